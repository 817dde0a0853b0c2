"""Particle-record and parameter layouts shared with include/sph_isph.h.

The record dtypes reproduce the reference's AoS structs part1/part2/part3
(class_Cuda_Particle_Array.cuh:11-112, Real = float, int_t = int): 152, 52 and
164 bytes.  ``SphParams`` mirrors ``sph_params``: the reference's k_vii/k_vif
tables (function_init.cuh:84-163) plus the constants the reference hard-wires.
"""
import ctypes

import numpy as np

PART1_FIELDS = [
    ("i_type", "<i4"), ("buffer_type", "<i4"), ("MOST_buffer", "<i4"), ("p_type", "<i4"),
    ("x", "<f4"), ("y", "<f4"), ("z", "<f4"),
    ("ux", "<f4"), ("uy", "<f4"), ("uz", "<f4"),
    ("m", "<f4"), ("h", "<f4"), ("temp", "<f4"), ("pres", "<f4"), ("pres0", "<f4"),
    ("rho", "<f4"), ("flt_s", "<f4"), ("enthalpy", "<f4"), ("concn", "<f4"),
    ("concentration", "<f4"),
    ("k_turb", "<f4"), ("e_turb", "<f4"),
    ("eli", "<f4"), ("vol", "<f4"),
    ("m_ref", "<f4"), ("h_ref", "<f4"),
    ("vis_t", "<f4"),
    ("fbx", "<f4"), ("fby", "<f4"), ("fbz", "<f4"),
    ("fmx", "<f4"), ("fmy", "<f4"), ("hmz", "<f4"),
    ("float1", "<f4"), ("float2", "<f4"), ("float3", "<f4"),
    ("ncell", "<i4"), ("source", "<i4"),
]
PART2_FIELDS = [
    ("rho_ref", "<f4"), ("SR", "<f4"),
    ("x0", "<f4"), ("y0", "<f4"), ("z0", "<f4"),
    ("ux0", "<f4"), ("uy0", "<f4"), ("uz0", "<f4"),
    ("rho0", "<f4"), ("drho0", "<f4"), ("temp0", "<f4"), ("concn0", "<f4"), ("enthalpy0", "<f4"),
]
PART3_FIELDS = [
    ("drho", "<f4"), ("dconcn", "<f4"), ("denthalpy", "<f4"),
    ("ftotalx", "<f4"), ("ftotaly", "<f4"), ("ftotalz", "<f4"), ("ftotal", "<f4"),
    ("fpx", "<f4"), ("fpy", "<f4"), ("fpz", "<f4"), ("fbody", "<f4"),
    ("dtemp", "<f4"), ("dk_turb", "<f4"), ("de_trub", "<f4"), ("cc", "<f4"),
    ("nx", "<f4"), ("ny", "<f4"), ("nz", "<f4"),
    ("Cm", "<f4", (3, 3)),
    ("inv_cm_xx", "<f4"), ("inv_cm_yy", "<f4"), ("inv_cm_zz", "<f4"),
    ("inv_cm_xy", "<f4"), ("inv_cm_yz", "<f4"), ("inv_cm_zx", "<f4"),
    ("Gxx", "<f4"), ("Gxy", "<f4"), ("Gyx", "<f4"), ("Gyy", "<f4"),
    ("L11", "<f4"), ("L12", "<f4"), ("L21", "<f4"), ("L22", "<f4"),
]

PART1 = np.dtype(PART1_FIELDS)
PART2 = np.dtype(PART2_FIELDS)
PART3 = np.dtype(PART3_FIELDS)
assert PART1.itemsize == 152 and PART2.itemsize == 52 and PART3.itemsize == 164

# k_vii / k_vif slot names, function_init.cuh:2-82
VII = dict(solver_type=0, dim=1, prop_table=2, kernel_type=3, time_type=4, open_boundary=5,
           flag_timestep_update=6, nb_cell_type=7, freq_filt=8, freq_mass_sum=9, freq_temp=10,
           freq_output=11, fp_solve=12, fv_solve=13, fg_solve=14, con_solve=15,
           boussinesq_solve=16, kgc_solve=17, turbulence_model=18, concn_solve=19,
           minIteration=20, maxIteration=21, nb_cell_number=22, num_part=23, NI=24, NJ=25,
           NK=26, count=27, num_cells=28, ngpu=29, calc_area=30, num_p2p=31, num_part2=32,
           switch_ptype=33, noslip_bc=34, apr_solv=35, h_change=36, freq_apr=37,
           freq_h_reset=38, num_blocks=39, freq_bapr=40, NBI=41, NBJ=42, NBK=43,
           structure_solv=44, atmos_stab=45, terrain_type=46)
VIF = dict(kappa=0, p_ref=1, dt=2, time=3, time_end=4, u_limit=5, drho_th=6, dp_th=7,
           p_relaxation=8, x_min=9, x_max=10, y_min=11, y_max=12, z_min=13, z_max=14,
           nd_ref=15, search_incr_factor=16, search_kappa=17, dcell=18, buffersize=19,
           dt_structure=20)

# Parameters.cuh codes
KERNELS = dict(Gaussian=0, Quintic=1, Quartic=2, Wendland2=3, Wendland4=4, Wendland6=5)
TURB = dict(Laminar=0, K_LM=1, K_E=2, HB=3, SSM=4, DDF=5)
EULER, PRE_COR = 0, 1
CLEARY, MONAGHAN = 1, 2
KGC = 1

PREC_MIXED, PREC_FP64 = 0, 1
PPE_REF_SWEEP, PPE_BICGSTAB, PPE_MIXED_IR, PPE_LEARNED, PPE_GMRES, PPE_IDRS = 0, 1, 2, 3, 4, 5

MAX_PROFILE = 32


class SphParams(ctypes.Structure):
    """ctypes mirror of ``sph_params`` (include/sph_isph.h)."""
    _fields_ = [
        ("vii", ctypes.c_int32 * 64),
        ("vif", ctypes.c_float * 32),
        ("cs_sgs", ctypes.c_double),
        ("l2", ctypes.c_double), ("l3", ctypes.c_double),
        ("l_left", ctypes.c_double), ("l_right", ctypes.c_double),
        ("outlet_probe_dx", ctypes.c_double),
        ("partner_tol", ctypes.c_double),
        ("ghost_tol", ctypes.c_double),
        ("ib_box", ctypes.c_double * 6),
        ("ib_face_tol", ctypes.c_double),
        ("most_z0", ctypes.c_double), ("most_z0h", ctypes.c_double),
        ("most_ghost_dz", ctypes.c_double),
        ("rho_air", ctypes.c_double),
        ("ibm_target_coeff", ctypes.c_double),
        ("visc_fluid", ctypes.c_double), ("visc_wall", ctypes.c_double),
        ("visc_marker", ctypes.c_double),
        ("av_alpha", ctypes.c_double), ("av_beta", ctypes.c_double), ("av_c0", ctypes.c_double),
        ("pressure_length", ctypes.c_double), ("ibm_length", ctypes.c_double),
        ("neumann_coeff", ctypes.c_double),
        ("t_ini", ctypes.c_double), ("t_con", ctypes.c_double),
        ("t_start", ctypes.c_double), ("t_con_t", ctypes.c_double),
        ("boundary_velocity", ctypes.c_double),
        ("n_profile", ctypes.c_int32),
        ("pad0", ctypes.c_int32),
        ("profile_z", ctypes.c_double * MAX_PROFILE),
        ("profile_u", ctypes.c_double * MAX_PROFILE),
        ("ppe_mode", ctypes.c_int32),
        ("ppe_max_iter", ctypes.c_int32),
        ("ppe_tol", ctypes.c_double),
        ("ppe_pin", ctypes.c_int32),
        ("recompute_gc", ctypes.c_int32),
        ("ppe_matrix_free", ctypes.c_int32),
        ("ppe_gmres_restart", ctypes.c_int32),
        ("ppe_refinement", ctypes.c_int32),
        ("ppe_coarse_block", ctypes.c_int32),
        ("ppe_warm_start", ctypes.c_int32),
        ("apr_max_level", ctypes.c_int32),
        ("outlet_bc", ctypes.c_int32),
        ("inlet_recycling", ctypes.c_int32),
        ("ppe_coarse_mode", ctypes.c_int32),
        ("ppe_pair_h", ctypes.c_int32),
        ("ppe_wide_index", ctypes.c_int32),
        ("recompute_pairs", ctypes.c_int32),
        ("pressure_force_form", ctypes.c_int32),
        ("ppe_coef_half", ctypes.c_int32),
        ("ppe_coarse_max", ctypes.c_int32),
        ("enthalpy_eqn", ctypes.c_int32),
        ("ppe_inner_tol", ctypes.c_double),
        ("apr_zone", ctypes.c_double),
        ("recycle_probe_x", ctypes.c_double), ("recycle_probe_y", ctypes.c_double),
        ("periodic_box", ctypes.c_double * 6),
    ]

    def seti(self, name, value):
        self.vii[VII[name]] = int(value)

    def setf(self, name, value):
        self.vif[VIF[name]] = float(value)

    def geti(self, name):
        return int(self.vii[VII[name]])

    def getf(self, name):
        return float(self.vif[VIF[name]])

    def copy(self):
        out = SphParams()
        ctypes.pointer(out)[0] = self
        return out


class PpeStats(ctypes.Structure):
    """ctypes mirror of ``sph_ppe_stats``."""
    _fields_ = [
        ("status", ctypes.c_int32), ("iterations", ctypes.c_int32),
        ("refinements", ctypes.c_int32), ("restarts", ctypes.c_int32),
        ("rel_residual", ctypes.c_double), ("solve_ms", ctypes.c_double),
        ("initial_residual", ctypes.c_double),
    ]


assert ctypes.sizeof(SphParams) == 1344, ctypes.sizeof(SphParams)

TABLE_SIZE = 50     # table_size, Parameters.cuh:66
TABLE_SLOTS = 10    # k_table_index / k_table_size, SOPHIA_gpu.cu:56-57


class PropTables(ctypes.Structure):
    """ctypes mirror of ``sph_prop_tables``: the property tables of read_table
    (function_init.cuh:724-905); table t spans entries index[t] ..
    index[t] + size[t] - 1 of each column and serves |p_type| = t."""
    _fields_ = [
        ("n_tables", ctypes.c_int32), ("n_data", ctypes.c_int32),
        ("index", ctypes.c_int32 * TABLE_SLOTS), ("size", ctypes.c_int32 * TABLE_SLOTS),
        ("T", ctypes.c_double * TABLE_SIZE), ("h", ctypes.c_double * TABLE_SIZE),
        ("k", ctypes.c_double * TABLE_SIZE), ("cp", ctypes.c_double * TABLE_SIZE),
        ("mu", ctypes.c_double * TABLE_SIZE),
    ]

    def column(self, name, t):
        """Entries of column `name` in table t."""
        a = np.ctypeslib.as_array(getattr(self, name))
        return a[self.index[t]:self.index[t] + self.size[t]].copy()

    @classmethod
    def from_columns(cls, tables):
        """Tables from a list (slot 0, 1, ...) of dicts of equal-length columns
        (T, h, k, cp, mu; missing ones 0), laid end to end as read_table
        lays them."""
        out = cls()
        at = 0
        for t, cols in enumerate(tables):
            n = len(next(iter(cols.values())))
            for name, v in cols.items():
                assert len(v) == n, name
                getattr(out, name)[at:at + n] = [float(x) for x in v]
            out.index[t], out.size[t] = at, n
            at += n
        out.n_tables, out.n_data = len(tables), at
        return out


assert ctypes.sizeof(PropTables) == 2088, ctypes.sizeof(PropTables)

BUFFER_PERIODIC_GHOST = 7   # buffer_type of a periodic ghost (sph_params.periodic_box)

OUTLET_DONOTHING = 0      # KERNEL_donothing_buffer3D (the shipped step)
OUTLET_EXTRAPOLATION = 1  # KERNEL_open_boundary_extrapolation_buffer3D
OUTLET_INOUT = 2          # KERNEL_inout_boundary3D


def params_from_bytes(b):
    """SphParams from stored bytes; fields appended since they were written
    (apr_zone, the recycling probe, the periodic box) read as 0."""
    buf = bytearray(ctypes.sizeof(SphParams))
    b = bytes(b)
    buf[:len(b)] = b[:len(buf)]
    return SphParams.from_buffer_copy(buf)
