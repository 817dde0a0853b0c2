"""Reference defaults and host-side domain set-up.

``default_params`` fills a ``SphParams`` the way the reference's solver input
does for an urban ISPH case (read_solv_input, function_init.cuh:166-463), and
sets the constants the reference hard-wires to the reference's values.
``domain_setup`` restates ISPH.cuh:83-97 and clc_num_cells
(functions_NNPS.cuh:533-546) in FP32, as the reference evaluates them.
"""
import numpy as np

from .layout import (KERNELS, PPE_MIXED_IR, PRE_COR, CLEARY, TURB, SphParams)

# Wall-model target profile of functions_IBM.cuh:289-304 (AIJ Case H), the
# table the reference uses for the IBM tangential target velocity.
CASEH_PROFILE_Z = (0.005, 0.01, 0.02, 0.04, 0.06, 0.08, 0.1, 0.12, 0.14, 0.16,
                   0.165, 0.17, 0.18, 0.19, 0.21, 0.23, 0.25, 0.3, 0.35, 0.4,
                   0.45, 0.5, 0.55, 0.6, 0.6528736, 0.7724136, 0.8390808, 0.8689656,
                   0.88046, 0.8919544)
CASEH_PROFILE_U = (2.745, 2.935, 3.175, 3.435, 3.627, 3.824, 4.021, 4.21, 4.362, 4.491,
                   4.502, 4.586, 4.606, 4.712, 4.854, 4.993, 5.132, 5.449, 5.782, 6.077,
                   6.338, 6.588, 6.693, 6.751, 6.751, 6.751, 6.751, 6.751, 6.751, 6.751)


def default_params(dt=1e-4, kernel="Wendland6", turbulence="SSM", viscous=CLEARY,
                   kappa=2.0, u_limit=50.0, open_boundary=1, noslip=1):
    """Solver settings of an urban ISPH run plus the reference constants."""
    p = SphParams()
    p.seti("solver_type", 1)          # ISPH
    p.seti("dim", 3)
    p.seti("kernel_type", KERNELS[kernel])
    p.seti("time_type", PRE_COR)
    p.seti("open_boundary", open_boundary)
    p.seti("freq_filt", 1)
    p.seti("freq_output", 100)
    p.seti("fp_solve", 1)
    p.seti("fv_solve", viscous)
    p.seti("fg_solve", 0)
    p.seti("kgc_solve", 0)
    p.seti("turbulence_model", TURB[turbulence])
    p.seti("noslip_bc", noslip)
    p.seti("ngpu", 1)
    p.setf("kappa", kappa)
    p.setf("dt", dt)
    p.setf("time", 0.0)
    p.setf("time_end", 1.0)
    p.setf("u_limit", u_limit)
    p.setf("dt_structure", dt)

    p.cs_sgs = 0.15
    p.l2, p.l3 = 0.028, 13.304
    p.l_left, p.l_right = -0.412, 0.412
    p.outlet_probe_dx = 0.008
    p.partner_tol = 0.001
    p.ghost_tol = 0.1
    for k, v in enumerate((0.764, 0.836, -0.036, 0.036, 0.0, 0.152)):
        p.ib_box[k] = v
    p.ib_face_tol = 1e-5
    p.most_z0, p.most_z0h = 1.0, 0.1
    p.most_ghost_dz = 5.0
    p.rho_air = 1.225
    p.ibm_target_coeff = 0.2
    p.visc_fluid, p.visc_wall, p.visc_marker = 1.8e-5, 1.0e-2, 1.0e-2
    p.av_alpha, p.av_beta, p.av_c0 = 0.05, 0.05, 30.0
    p.pressure_length, p.ibm_length, p.neumann_coeff = 1.0, 0.5, 2.0
    p.t_ini, p.t_con, p.t_start, p.t_con_t = 300.0, 300.0, 0.0, 10.0
    p.boundary_velocity = 1.0
    set_profile(p, CASEH_PROFILE_Z, CASEH_PROFILE_U)
    p.ppe_mode = PPE_MIXED_IR
    p.ppe_max_iter = 2000
    p.ppe_tol = 1e-6
    p.ppe_pin = 1
    p.recompute_gc = 0
    p.ppe_inner_tol = 1e-3
    p.recycle_probe_x, p.recycle_probe_y = 600.0, 0.0   # functions_MOST.cuh:316
    return p


def set_profile(p, z, u):
    z = list(z)
    u = list(u)
    assert 2 <= len(z) == len(u) <= 32
    p.n_profile = len(z)
    for k in range(len(z)):
        p.profile_z[k] = z[k]
        p.profile_u[k] = u[k]


def domain_setup(p, P1):
    """ISPH.cuh:83-97: min/max, dcell, NI/NJ/NK, num_cells (FP32 arithmetic)."""
    f = np.float32
    n = len(P1)
    # find_minmax (function_init.cuh:678-708) scans records 0..n-2 only
    sl = slice(0, max(n - 1, 1))
    xs, ys, zs = P1["x"][sl], P1["y"][sl], P1["z"][sl]
    x_min, x_max = min(f(P1["x"][0]), xs.min()), max(f(P1["x"][0]), xs.max())
    y_min, y_max = min(f(P1["y"][0]), ys.min()), max(f(P1["y"][0]), ys.max())
    z_min, z_max = min(f(P1["z"][0]), zs.min()), max(f(P1["z"][0]), zs.max())
    kappa = f(p.getf("kappa"))
    h0 = f(P1["h_ref"][0])
    dcell = f(f(f(f(1.1) * kappa) * h0) / f(2.0))
    ni = int(f((x_max - x_min) / dcell)) + 1
    nj = int(f((y_max - y_min) / dcell)) + 1
    nk = int(f((z_max - z_min) / dcell)) + 1
    p.setf("x_min", x_min); p.setf("x_max", x_max)
    p.setf("y_min", y_min); p.setf("y_max", y_max)
    p.setf("z_min", z_min); p.setf("z_max", z_max)
    p.setf("search_incr_factor", 1.0)
    p.setf("search_kappa", kappa)
    p.setf("dcell", dcell)
    p.seti("NI", ni); p.seti("NJ", nj); p.seti("NK", nk)
    p.seti("num_cells", ni * nj * nk + 1)
    p.seti("num_part", n)
    p.seti("num_part2", n)
    return p
