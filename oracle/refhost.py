"""ctypes driver for oracle/_ref/libsophia_ref.so (test infrastructure only).

The library is the reference's own device code compiled for the host by
oracle/Makefile (see ref_shim.cpp).  ``RefHost`` keeps the reference's arrays
(dev_P1, dev_SP1, dev_P2, dev_SP2, dev_P3, g_idx, p_idx, g_str, g_end of
ISPH_Calc.cuh:327-344) as numpy records and advances them with ref_step,
the host restatement of SOPHIA_single_ISPH's launch sequence.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libsophia_ref.so")

# host builds of the reference: as shipped (None), and with the pressure
# force's commented-out difference form in place of its active line ("dp")
VARIANTS = {None: LIB_PATH, "dp": os.path.join(HERE, "_ref", "libsophia_ref_dp.so"),
            "enth": os.path.join(HERE, "_ref", "libsophia_ref_enth.so")}
_libs = {}


def available(variant=None):
    return os.path.exists(VARIANTS[variant])


def lib(variant=None):
    if variant not in _libs:
        if not available(variant):
            raise FileNotFoundError(f"{VARIANTS[variant]} not built (make -C oracle ref ref_dp ref_enth)")
        L = ctypes.CDLL(VARIANTS[variant])
        vp = ctypes.c_void_p
        L.ref_set_params.argtypes = [vp, vp]
        L.ref_get_params.argtypes = [vp, vp]
        L.ref_domain_setup.argtypes = [vp, ctypes.c_int]
        L.ref_nnps.argtypes = [vp] * 8
        L.ref_step.argtypes = [vp] * 9 + [ctypes.c_int, ctypes.c_float, ctypes.c_int]
        L.ref_set_parallel.argtypes = [ctypes.c_int]
        L.ref_set_boundary_variant.argtypes = [ctypes.c_int] * 3
        L.ref_num_threads.restype = ctypes.c_int
        _libs[variant] = L
    return _libs[variant]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def read_table(path, variant=None):
    """The reference's read_table on `path` (and its upload to the arrays
    the device code reads): {"T", "h", "k", "cp", "mu"} as stored in Real
    (table_size entries each), index and size per slot."""
    L = lib(variant)
    L.ref_read_table.argtypes = [ctypes.c_char_p] + [ctypes.c_void_p] * 3
    L.ref_read_table.restype = None
    cols = np.zeros((5, 50), np.float64)
    index = np.zeros(10, np.int32)
    size = np.zeros(10, np.int32)
    L.ref_read_table(str(path).encode(), _p(cols), _p(index), _p(size))
    out = dict(zip(("T", "h", "k", "cp", "mu"), cols))
    out["index"], out["size"] = index, size
    return out


class RefHost:
    """Reference step on the host, one instance per deck."""

    def __init__(self, P1, params, parallel=True, variant=None):
        from sph_b200.layout import PART2, PART3
        self.L = L = lib(variant)
        self.params = params.copy()
        self.n = len(P1)
        L.ref_set_parallel(1 if parallel else 0)
        vii = np.ctypeslib.as_array(self.params.vii).copy()
        vif = np.ctypeslib.as_array(self.params.vif).copy()
        L.ref_set_params(_p(vii), _p(vif))
        L.ref_set_boundary_variant(int(self.params.outlet_bc), int(self.params.inlet_recycling), 1)
        self.P1 = np.array(P1, copy=True)
        self.SP1 = np.zeros_like(self.P1)
        self.P2 = np.zeros(self.n, dtype=PART2)
        self.SP2 = np.zeros(self.n, dtype=PART2)
        self.P3 = np.zeros(self.n, dtype=PART3)
        nc = self.params.geti("num_cells")
        self.g_idx = np.zeros(self.n, np.int32)
        self.p_idx = np.zeros(self.n, np.int32)
        self.g_str = np.full(nc + 1, -1, np.int32)
        self.g_end = np.zeros(nc + 1, np.int32)
        self.count = self.params.geti("count")
        self.time = np.float32(self.params.getf("time"))

    def temp_to_enthalpy(self):
        """The reference's KERNEL_clc_TemptoEnthalpy on the records (P1, P2)."""
        self.L.ref_temp_to_enthalpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        self.L.ref_temp_to_enthalpy(_p(self.P1), _p(self.P2), self.n)

    def enthalpy_to_temp(self):
        """The reference's KERNEL_clc_EnthalpytoTemp on the records (P1)."""
        self.L.ref_enthalpy_to_temp.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self.L.ref_enthalpy_to_temp(_p(self.P1), self.n)

    def _load_params(self):
        vii = np.ctypeslib.as_array(self.params.vii).copy()
        vif = np.ctypeslib.as_array(self.params.vif).copy()
        self.L.ref_set_params(_p(vii), _p(vif))
        self.L.ref_set_boundary_variant(int(self.params.outlet_bc), int(self.params.inlet_recycling), 0)

    def step(self, nsteps=1, ppe_snapshot=True):
        L = self.L
        self._load_params()
        for _ in range(nsteps):
            L.ref_step(_p(self.P1), _p(self.SP1), _p(self.P2), _p(self.SP2), _p(self.P3),
                       _p(self.g_idx), _p(self.p_idx), _p(self.g_str), _p(self.g_end),
                       int(self.count), float(self.time), 1 if ppe_snapshot else 0)
            # ISPH_Calc.cuh:496-497
            self.time = np.float32(self.time + np.float32(self.params.getf("dt")))
            self.count += 1

    def nnps(self):
        """Step-0 NNPS only (ISPH_Calc.cuh:20-45) on a copy of P1."""
        L = self.L
        self._load_params()
        P1 = np.array(self.P1, copy=True)
        P2 = np.array(self.P2, copy=True)
        SP1 = np.zeros_like(P1)
        SP2 = np.zeros_like(P2)
        L.ref_nnps(_p(P1), _p(P2), _p(SP1), _p(SP2), _p(self.g_idx), _p(self.p_idx),
                   _p(self.g_str), _p(self.g_end))
        return SP1, self.g_idx.copy(), self.p_idx.copy(), self.g_str.copy(), self.g_end.copy()


APR_LIB_PATH = os.path.join(HERE, "_ref", "libsophia_ref_apr.so")
_apr_lib = None


def apr_available():
    return os.path.exists(APR_LIB_PATH)


def apr_lib():
    """The reference's APR kernels compiled for the host (ref_apr_shim.cpp)."""
    global _apr_lib
    if _apr_lib is None:
        L = ctypes.CDLL(APR_LIB_PATH)
        vp = ctypes.c_void_p
        L.refapr_set_params.argtypes = [vp, vp]
        L.refapr_condition.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp]
        L.refapr_split.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]
        _apr_lib = L
    return _apr_lib


def ref_apr_pass(P, g_str, g_end, params, target, family, first_free):
    """The reference's condition, numbering and split on a sorted state:
    returns (apr_cond, apr_cell, records after the split, M_num, blood_index)."""
    L = apr_lib()
    vii = np.ctypeslib.as_array(params.vii).copy()
    vif = np.ctypeslib.as_array(params.vif).copy()
    L.refapr_set_params(_p(vii), _p(vif))
    n = len(P)
    nc = params.geti("num_cells")
    R = np.ascontiguousarray(P.copy())
    M = np.ascontiguousarray(target, np.float32)
    B = np.ascontiguousarray(family, np.int32)
    gs = np.ascontiguousarray(g_str, np.int32)
    ge = np.ascontiguousarray(g_end, np.int32)
    cond = np.zeros(n, np.int32)
    cell = np.zeros(nc, np.int32)
    L.refapr_condition(_p(R), n, _p(M), _p(B), _p(gs), _p(ge), _p(cond), _p(cell))
    Mo = np.zeros(n, np.float32)
    Bo = np.zeros(n, np.int32)
    # KERNEL_cell_APR_3D writes children up to first_free + 8 * (splits + 1)
    # without a bound: refuse states without that room
    if first_free + 8 * (int((cell > 0).sum()) + 1) > n:
        raise ValueError("not enough free records for the reference's split")
    num_part = params.geti("num_part")
    L.refapr_split(_p(R), n, int(first_free - num_part), _p(gs), _p(ge), _p(Mo), _p(Bo))
    return cond, cell, R, Mo, Bo
