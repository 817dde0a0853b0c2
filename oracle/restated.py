"""ctypes driver for oracle/lib/libsph_oracle.so, the CPU restatement of the
reference ISPH step (test infrastructure only; see sph_oracle.cpp)."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsph_oracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle)")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.orc_create.argtypes = [vp, ctypes.c_int]
        L.orc_create.restype = vp
        L.orc_destroy.argtypes = [vp]
        L.orc_set_params.argtypes = [vp, vp]
        L.orc_upload.argtypes = [vp, vp, ctypes.c_int]
        L.orc_nnps.argtypes = [vp]
        L.orc_export_nnps.argtypes = [vp] * 5
        L.orc_nnz.argtypes = [vp]
        L.orc_nnz.restype = ctypes.c_int64
        L.orc_export_neighbors.argtypes = [vp] * 3
        L.orc_step.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, vp, vp]
        L.orc_pin_row.argtypes = [vp]
        L.orc_download.argtypes = [vp] * 4
        L.orc_set_tables.argtypes = [vp, vp]
        L.orc_temp_to_enthalpy.argtypes = [vp, ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Restated:
    """One oracle instance (precision 0 = FP32 as the reference, 1 = FP64)."""

    def __init__(self, P1, params, precision=0):
        L = lib()
        self.params = params.copy()
        self.n = len(P1)
        self.h = L.orc_create(ctypes.byref(self.params), precision)
        P = np.ascontiguousarray(P1)
        L.orc_upload(self.h, _p(P), self.n)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_params(self, params):
        self.params = params.copy()
        lib().orc_set_params(self.h, ctypes.byref(self.params))

    def nnps(self):
        lib().orc_nnps(self.h)

    def export_nnps(self):
        nc = self.params.geti("num_cells") + 1
        g_idx = np.zeros(self.n, np.int32); p_idx = np.zeros(self.n, np.int32)
        g_str = np.zeros(nc, np.int32); g_end = np.zeros(nc, np.int32)
        lib().orc_export_nnps(self.h, _p(g_idx), _p(p_idx), _p(g_str), _p(g_end))
        return g_idx, p_idx, g_str, g_end

    def neighbors(self):
        L = lib()
        nnz = L.orc_nnz(self.h)
        off = np.zeros(self.n + 1, np.int64)
        lst = np.zeros(max(nnz, 1), np.int32)
        L.orc_export_neighbors(self.h, _p(off), _p(lst))
        return off, lst[:nnz]

    def step(self, nsteps=1, mode=0, tol=1e-8, maxit=5000):
        rr = ctypes.c_double(0)
        it = ctypes.c_int(0)
        st = 0
        for _ in range(nsteps):
            st = lib().orc_step(self.h, mode, tol, maxit, ctypes.byref(rr), ctypes.byref(it))
        return st, rr.value, it.value

    def set_tables(self, tables):
        """Property tables (a PropTables) for htoT with vii[prop_table] = 1."""
        lib().orc_set_tables(self.h, ctypes.byref(tables))

    def temp_to_enthalpy(self):
        """enthalpy = enthalpy0 = Ttoh(temp, p_type) for every record but i_type 3."""
        lib().orc_temp_to_enthalpy(self.h, 0)

    def enthalpy_to_temp(self):
        """temp = htoT(enthalpy, p_type) for every record but i_type 3."""
        lib().orc_temp_to_enthalpy(self.h, 1)

    def pin_row(self):
        return lib().orc_pin_row(self.h)

    def download(self):
        from sph_b200.layout import PART1, PART2, PART3
        P1 = np.zeros(self.n, PART1); P2 = np.zeros(self.n, PART2); P3 = np.zeros(self.n, PART3)
        lib().orc_download(self.h, _p(P1), _p(P2), _p(P3))
        return P1, P2, P3
