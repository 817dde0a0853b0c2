"""ctypes binding of lib/libsph_b200.so (include/sph_isph.h).

``Simulation`` is the host-side mirror of the reference's step driver
(SOPHIA_single_ISPH, ISPH_Calc.cuh:4-233): it owns one device context and
exposes the reference phases (NNPS, interaction, PPE, time update) over the
reference's part1/part2/part3 records.  There is no CPU fallback: loading the
library or creating a context on a machine without the CUDA build or a GPU
raises.
"""
import ctypes
import os

import numpy as np

from .layout import PART1, PART2, PART3, PpeStats, PropTables, SphParams

ML_NPARAM = 5569   # SPH_ML_NPARAM

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libsph_b200.so")

# every entry point declared in include/sph_isph.h
SYMBOLS = (
    "sph_params_init", "sph_domain_setup", "sph_create", "sph_destroy", "sph_set_params",
    "sph_upload", "sph_upload_state", "sph_download", "sph_nnps", "sph_nnps_export",
    "sph_neighbors_export", "sph_interaction", "sph_ppe", "sph_time_update", "sph_step",
    "sph_diagnostics", "sph_last_phase_ms", "sph_launch_count", "sph_step_graph_count", "sph_operator_counts", "sph_status_string",
    "sph_last_error", "sph_profile", "sph_set_pair_block", "sph_operator_stats", "sph_operator_bytes", "sph_nnps_sort_noalloc",
    "sph_ml_collect", "sph_ml_samples", "sph_ml_train", "sph_ml_set_weights", "sph_ml_get_weights",
    "sph_ml_grad", "sph_ml_predict_samples",
    "sph_batch_create", "sph_batch_destroy", "sph_batch_step", "sph_batch_set_workers", "sph_batch_autotune",
    "sph_batch_autotune_shapes",
    "sph_batch_case", "sph_batch_particles", "sph_apr", "sph_apr_state", "sph_set_ib_boxes", "sph_read_deck", "sph_write_vtk",
    "sph_read_solv", "sph_initial_records", "sph_read_table", "sph_set_prop_tables",
    "sph_energy_convert",
)

_lib = None


class SphError(RuntimeError):
    def __init__(self, where, status):
        L = lib()
        msg = L.sph_status_string(status).decode()
        detail = L.sph_last_error().decode()
        super().__init__(f"{where}: {msg} ({status}) {detail}")
        self.status = status


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: build it with urban-sph_a100_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        L.sph_params_init.argtypes = [vp]
        L.sph_domain_setup.argtypes = [vp, vp, i32]
        L.sph_create.argtypes = [vp, i32, i32, vp, ctypes.POINTER(vp)]
        L.sph_destroy.argtypes = [vp]
        L.sph_destroy.restype = None
        L.sph_set_params.argtypes = [vp, vp]
        L.sph_upload.argtypes = [vp, vp, vp, i32]
        L.sph_upload_state.argtypes = [vp, vp, i32]
        L.sph_download.argtypes = [vp, vp, vp, vp]
        L.sph_nnps.argtypes = [vp]
        L.sph_nnps_export.argtypes = [vp, vp, vp, vp, vp]
        L.sph_neighbors_export.argtypes = [vp, vp, vp, ctypes.POINTER(i64)]
        L.sph_interaction.argtypes = [vp]
        L.sph_ppe.argtypes = [vp, vp]
        L.sph_time_update.argtypes = [vp]
        L.sph_step.argtypes = [vp, i32, vp]
        L.sph_diagnostics.argtypes = [vp, vp, vp, vp]
        L.sph_last_phase_ms.argtypes = [vp, vp]
        L.sph_launch_count.argtypes = [vp]
        L.sph_launch_count.restype = i64
        L.sph_step_graph_count.argtypes = [vp]
        L.sph_step_graph_count.restype = i64
        L.sph_operator_counts.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.sph_operator_counts.restype = ctypes.c_int
        L.sph_status_string.argtypes = [i32]
        L.sph_status_string.restype = ctypes.c_char_p
        L.sph_last_error.restype = ctypes.c_char_p
        L.sph_profile.argtypes = [vp, i32]
        L.sph_set_pair_block.argtypes = [vp, i32]
        L.sph_operator_stats.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double), i32]
        L.sph_operator_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.sph_nnps_sort_noalloc.argtypes = [vp, vp, vp, vp, vp, i32, vp, vp, vp, vp, vp]
        f32p = ctypes.POINTER(ctypes.c_float)
        L.sph_ml_collect.argtypes = [vp, i32]
        L.sph_ml_samples.argtypes = [vp, i64, i64, vp, vp, ctypes.POINTER(i64)]
        L.sph_ml_train.argtypes = [vp, i32, i32, ctypes.c_float, ctypes.c_uint64, f32p]
        L.sph_ml_set_weights.argtypes = [vp, vp]
        L.sph_ml_get_weights.argtypes = [vp, vp]
        L.sph_ml_grad.argtypes = [vp, i64, i32, f32p, vp]
        L.sph_ml_predict_samples.argtypes = [vp, i64, i32, vp]
        L.sph_batch_create.argtypes = [i32, vp, vp, vp, i32, i32, ctypes.POINTER(vp)]
        L.sph_batch_destroy.argtypes = [vp]
        L.sph_batch_destroy.restype = None
        L.sph_batch_step.argtypes = [vp, i32, vp]
        L.sph_batch_set_workers.argtypes = [vp, i32]
        L.sph_batch_autotune.argtypes = [vp, i32, ctypes.POINTER(i32), ctypes.POINTER(ctypes.c_double)]
        L.sph_batch_autotune_shapes.argtypes = [vp, i32, ctypes.POINTER(i32), ctypes.POINTER(i32),
                                                ctypes.POINTER(ctypes.c_double)]
        L.sph_batch_case.argtypes = [vp, i32, ctypes.POINTER(vp)]
        L.sph_batch_particles.argtypes = [vp]
        L.sph_batch_particles.restype = i64
        L.sph_apr.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        L.sph_apr_state.argtypes = [vp, vp, vp, ctypes.POINTER(i32)]
        L.sph_set_ib_boxes.argtypes = [vp, vp, i32]
        L.sph_read_deck.argtypes = [ctypes.c_char_p, vp, i32, ctypes.POINTER(i32)]
        L.sph_read_solv.argtypes = [ctypes.c_char_p, vp, vp, ctypes.POINTER(i32)]
        L.sph_initial_records.argtypes = [vp, vp, i32, vp, i32, ctypes.c_double, ctypes.c_double]
        L.sph_read_table.argtypes = [ctypes.c_char_p, vp]
        L.sph_set_prop_tables.argtypes = [vp, vp]
        L.sph_energy_convert.argtypes = [vp, i32]
        L.sph_write_vtk.argtypes = [ctypes.c_char_p, vp, vp, vp, i32, ctypes.POINTER(ctypes.c_char_p), i32]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def records_arg(a, dtype, n=None):
    """(pointer, keep-alive, count) of a record array for the upload and
    download calls.  Device arrays (anything with __cuda_array_interface__,
    e.g. a CUDA torch tensor of uint8 or a CuPy array) pass their device
    pointer as they are, which the C ABI takes as well as host memory; they
    must be C-contiguous and hold a whole number of records (n of them when
    n is given).  Host arrays are made contiguous records of `dtype`."""
    cai = getattr(a, "__cuda_array_interface__", None)
    if cai is not None:
        shape = tuple(cai["shape"])
        item = np.dtype(cai["typestr"]).itemsize
        strides = cai.get("strides")
        if strides is not None:
            want, s_ = [], item
            for d in reversed(shape):
                want.append(s_)
                s_ *= d
            if tuple(strides) != tuple(reversed(want)):
                raise ValueError("device records must be C-contiguous")
        nbytes = int(np.prod(shape, dtype=np.int64)) * item
        if nbytes % dtype.itemsize:
            raise ValueError("device array of %d bytes is not a whole number of %d-byte records"
                             % (nbytes, dtype.itemsize))
        count = nbytes // dtype.itemsize
        if n is not None and count != n:
            raise ValueError("device array holds %d records, %d expected" % (count, n))
        return ctypes.c_void_p(int(cai["data"][0])), a, count
    arr = np.ascontiguousarray(a, dtype=dtype)
    if n is not None and len(arr) != n:
        raise ValueError("array holds %d records, %d expected" % (len(arr), n))
    return _p(arr), arr, len(arr)


def _check(where, st, ok=(0,)):
    if st not in ok and st < 0:
        raise SphError(where, st)
    return st


def params_init():
    p = SphParams()
    _check("sph_params_init", lib().sph_params_init(ctypes.byref(p)))
    return p


def domain_setup(p, P1):
    P1 = np.ascontiguousarray(P1, dtype=PART1)
    _check("sph_domain_setup", lib().sph_domain_setup(ctypes.byref(p), _p(P1), len(P1)))
    return p


class Simulation:
    """One device context: the reference's dev_P1/SP1/P2/SP2/P3 and NNPS arrays."""

    def __init__(self, params, precision=0, device=0, stream=None):
        self.params = params.copy()
        self.n = self.params.geti("num_part2")
        self.num_cells = self.params.geti("num_cells")
        h = ctypes.c_void_p()
        _check("sph_create", lib().sph_create(ctypes.byref(self.params), int(precision), int(device),
                                              stream, ctypes.byref(h)))
        self.h = h
        self.precision = precision
        self.last_stats = PpeStats()

    def close(self):
        if getattr(self, "h", None):
            lib().sph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        self.params = params.copy()
        _check("sph_set_params", lib().sph_set_params(self.h, ctypes.byref(self.params)))

    def upload(self, P1, P2=None):
        p1, keep1, n = records_arg(P1, PART1)
        p2, keep2 = (None, None) if P2 is None else records_arg(P2, PART2, n)[:2]
        _check("sph_upload", lib().sph_upload(self.h, p1, p2, n))

    def upload_state(self, P1):
        p1, keep1, n = records_arg(P1, PART1)
        _check("sph_upload_state", lib().sph_upload_state(self.h, p1, n))

    def download(self, want=(1, 2, 3)):
        P1 = np.zeros(self.n, PART1) if 1 in want else None
        P2 = np.zeros(self.n, PART2) if 2 in want else None
        P3 = np.zeros(self.n, PART3) if 3 in want else None
        _check("sph_download", lib().sph_download(self.h, _p(P1), _p(P2), _p(P3)))
        return P1, P2, P3

    def download_into(self, P1, P2=None, P3=None):
        """Downloads into caller arrays: host records (numpy, contiguous) or
        device arrays (__cuda_array_interface__) of self.n records each."""
        ptrs = []
        for a, dt in ((P1, PART1), (P2, PART2), (P3, PART3)):
            if a is None:
                ptrs.append(None)
                continue
            if getattr(a, "__cuda_array_interface__", None) is None and not (
                    isinstance(a, np.ndarray) and a.flags.c_contiguous and a.dtype == dt):
                raise ValueError("download_into needs contiguous %s records or a device array" % dt)
            ptrs.append(records_arg(a, dt, self.n)[0])
        _check("sph_download", lib().sph_download(self.h, *ptrs))

    def nnps(self):
        _check("sph_nnps", lib().sph_nnps(self.h))

    def export_nnps(self):
        g_idx = np.zeros(self.n, np.int32); p_idx = np.zeros(self.n, np.int32)
        g_str = np.zeros(self.num_cells + 1, np.int32); g_end = np.zeros(self.num_cells + 1, np.int32)
        _check("sph_nnps_export", lib().sph_nnps_export(self.h, _p(g_idx), _p(p_idx), _p(g_str), _p(g_end)))
        return g_idx, p_idx, g_str, g_end

    def neighbors(self):
        nnz = ctypes.c_int64(0)
        off = np.zeros(self.n + 1, np.int64)
        _check("sph_neighbors_export", lib().sph_neighbors_export(self.h, _p(off), None, ctypes.byref(nnz)))
        lst = np.zeros(max(nnz.value, 1), np.int32)
        _check("sph_neighbors_export", lib().sph_neighbors_export(self.h, _p(off), _p(lst), ctypes.byref(nnz)))
        return off, lst[:nnz.value]

    def interaction(self):
        _check("sph_interaction", lib().sph_interaction(self.h))

    def ppe(self):
        st = PpeStats()
        _check("sph_ppe", lib().sph_ppe(self.h, ctypes.byref(st)))
        self.last_stats = st
        return st

    def time_update(self):
        _check("sph_time_update", lib().sph_time_update(self.h))

    def step(self, nsteps=1):
        st = PpeStats()
        _check("sph_step", lib().sph_step(self.h, int(nsteps), ctypes.byref(st)))
        self.last_stats = st
        return st

    def diagnostics(self):
        a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        _check("sph_diagnostics", lib().sph_diagnostics(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def phase_ms(self):
        ms = np.zeros(4, np.float32)
        _check("sph_last_phase_ms", lib().sph_last_phase_ms(self.h, _p(ms)))
        return ms

    def launches(self):
        return int(lib().sph_launch_count(self.h))

    def operator_counts(self):
        """Rows, fluid-row entries, Neumann rows, Neumann entries, cells of the pressure operator, and
        whether it reads 16-bit neighbour codes."""
        a = (ctypes.c_int64 * 6)()
        _check("sph_operator_counts", lib().sph_operator_counts(self.h, a))
        return {"rows": a[0], "entries": a[1], "neumann_rows": a[2], "neumann_entries": a[3], "cells": a[4],
                "codes16": bool(a[5])}

    def set_prop_tables(self, tables):
        """Uploads property tables (a PropTables, e.g. from read_table) for the
        enthalpy form's htoT with vii[prop_table] = 1."""
        _check("sph_set_prop_tables", lib().sph_set_prop_tables(self.h, ctypes.byref(tables)))

    def enthalpy_from_temperature(self):
        """enthalpy = enthalpy0 = Ttoh(temp, p_type) on the current records
        (the reference's KERNEL_clc_TemptoEnthalpy)."""
        _check("sph_energy_convert", lib().sph_energy_convert(self.h, 1))

    def temperature_from_enthalpy(self):
        """temp = htoT(enthalpy, p_type) on the current records (the
        reference's KERNEL_clc_EnthalpytoTemp)."""
        _check("sph_energy_convert", lib().sph_energy_convert(self.h, 0))

    def graph_steps(self):
        """Steps run as a replay of the whole-step graph."""
        return int(lib().sph_step_graph_count(self.h))

    def set_pair_block(self, threads):
        _check("sph_set_pair_block", lib().sph_set_pair_block(self.h, int(threads)))

    def profile(self, enable=True):
        _check("sph_profile", lib().sph_profile(self.h, 1 if enable else 0))

    def set_ib_boxes(self, boxes):
        b = np.ascontiguousarray(boxes, np.float64).reshape(-1, 6)
        _check("sph_set_ib_boxes", lib().sph_set_ib_boxes(self.h, _p(b), len(b)))

    def apr(self):
        a, b = ctypes.c_int32(0), ctypes.c_int32(0)
        _check("sph_apr", lib().sph_apr(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    # ---- learned warm start ----

    def apr_state(self):
        """(family, target level, families merged by the last pass) per record."""
        fam = np.zeros(self.n, np.int32)
        tgt = np.zeros(self.n, np.float32)
        nm = ctypes.c_int32(0)
        _check("sph_apr_state", lib().sph_apr_state(self.h, _p(fam), _p(tgt), ctypes.byref(nm)))
        return fam, tgt, nm.value
    def ml_collect(self, every):
        _check("sph_ml_collect", lib().sph_ml_collect(self.h, int(every)))

    def ml_samples(self, first=0, rows=None):
        cnt = ctypes.c_int64(0)
        _check("sph_ml_samples", lib().sph_ml_samples(self.h, 0, 0, None, None, ctypes.byref(cnt)))
        rows = cnt.value - first if rows is None else rows
        X = np.zeros((rows, 32), np.uint16)
        t = np.zeros(rows, np.float32)
        if rows > 0:
            _check("sph_ml_samples", lib().sph_ml_samples(self.h, first, rows, _p(X), _p(t), ctypes.byref(cnt)))
        return X, t

    def ml_train(self, epochs, batch, lr, seed=0):
        loss = ctypes.c_float(0)
        _check("sph_ml_train", lib().sph_ml_train(self.h, int(epochs), int(batch), float(lr), int(seed),
                                                  ctypes.byref(loss)))
        return loss.value

    def ml_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == ML_NPARAM
        _check("sph_ml_set_weights", lib().sph_ml_set_weights(self.h, _p(w)))

    def ml_get_weights(self):
        w = np.zeros(ML_NPARAM, np.float32)
        _check("sph_ml_get_weights", lib().sph_ml_get_weights(self.h, _p(w)))
        return w

    def ml_grad(self, first, rows):
        loss = ctypes.c_float(0)
        g = np.zeros(ML_NPARAM, np.float32)
        _check("sph_ml_grad", lib().sph_ml_grad(self.h, int(first), int(rows), ctypes.byref(loss), _p(g)))
        return loss.value, g

    def ml_predict_samples(self, first, rows):
        y = np.zeros(rows, np.float32)
        _check("sph_ml_predict_samples", lib().sph_ml_predict_samples(self.h, int(first), int(rows), _p(y)))
        return y

    def operator_stats(self, reset=True):
        n = ctypes.c_int64(0)
        ms = ctypes.c_double(0)
        by = ctypes.c_double(0)
        _check("sph_operator_stats", lib().sph_operator_stats(self.h, ctypes.byref(n), ctypes.byref(ms),
                                                              ctypes.byref(by), 1 if reset else 0))
        return n.value, ms.value, by.value

    def operator_bytes(self):
        """(stored, index_rule) bytes of one operator launch."""
        a = ctypes.c_double(0)
        b = ctypes.c_double(0)
        _check("sph_operator_bytes", lib().sph_operator_bytes(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value


class Batch:
    """Ensemble of independent cases on one GPU (sph_batch_*)."""

    def __init__(self, cases, precision=0, device=0):
        self._P = [np.ascontiguousarray(P, dtype=PART1) for P, _ in cases]
        self._params = (SphParams * len(cases))(*[p for _, p in cases])
        ptrs = (ctypes.c_void_p * len(cases))(*[P.ctypes.data for P in self._P])
        ns = np.array([len(P) for P in self._P], np.int32)
        h = ctypes.c_void_p()
        _check("sph_batch_create", lib().sph_batch_create(len(cases), self._params, ptrs, _p(ns), int(precision),
                                                          int(device), ctypes.byref(h)))
        self.h = h
        self.n = ns

    def close(self):
        if getattr(self, "h", None):
            lib().sph_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, nsteps=1):
        st = (PpeStats * len(self.n))()
        _check("sph_batch_step", lib().sph_batch_step(self.h, int(nsteps), st))
        return list(st)

    def set_workers(self, w):
        _check("sph_batch_set_workers", lib().sph_batch_set_workers(self.h, int(w)))

    def autotune(self, probe_steps=1):
        w, ms = ctypes.c_int32(0), ctypes.c_double(0)
        _check("sph_batch_autotune", lib().sph_batch_autotune(self.h, int(probe_steps), ctypes.byref(w), ctypes.byref(ms)))
        return w.value, ms.value

    def autotune_shapes(self, probe_steps=1):
        """(workers, pair-pass threads per block, ms per step) of the fastest probe."""
        w, t, ms = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0)
        _check("sph_batch_autotune_shapes", lib().sph_batch_autotune_shapes(self.h, int(probe_steps), ctypes.byref(w),
                                                                            ctypes.byref(t), ctypes.byref(ms)))
        return w.value, t.value, ms.value

    def download(self, k):
        c = ctypes.c_void_p()
        _check("sph_batch_case", lib().sph_batch_case(self.h, int(k), ctypes.byref(c)))
        P1 = np.zeros(int(self.n[k]), PART1)
        _check("sph_download", lib().sph_download(c, _p(P1), None, None))
        return P1

    def particles(self):
        return int(lib().sph_batch_particles(self.h))


def read_deck(path):
    """Records of a particle deck in the reference's input format."""
    n = ctypes.c_int32(0)
    p = str(path).encode()
    _check("sph_read_deck", lib().sph_read_deck(p, None, 0, ctypes.byref(n)))
    P = np.zeros(n.value, PART1)
    _check("sph_read_deck", lib().sph_read_deck(p, _p(P), len(P), ctypes.byref(n)))
    return P


def write_vtk(path, P1, labels, P2=None, P3=None):
    """The reference's binary VTK of the records (labels as in its solv.txt)."""
    arr = (ctypes.c_char_p * len(labels))(*[l.encode() for l in labels])
    P1 = np.ascontiguousarray(P1, dtype=PART1)
    _check("sph_write_vtk", lib().sph_write_vtk(str(path).encode(), _p(P1), _p(P2), _p(P3), len(P1), arr, len(labels)))


def read_solv(path, params=None):
    """Parameters and plot labels from a solver input file in the reference's format."""
    p = params.copy() if params is not None else params_init()
    labels = ctypes.create_string_buffer(400)
    n = ctypes.c_int32(0)
    _check("sph_read_solv", lib().sph_read_solv(str(path).encode(), ctypes.byref(p), labels, ctypes.byref(n)))
    raw = labels.raw
    return p, [raw[20 * k:20 * k + 20].split(b"\0")[0].decode() for k in range(min(n.value, 20))]


def read_table(path):
    """Property tables from a file in the reference's data.txt format."""
    t = PropTables()
    _check("sph_read_table", lib().sph_read_table(str(path).encode(), ctypes.byref(t)))
    return t


CASEH_L4 = 2210.0          # functions_NNPS.cuh:7
CASEH_L_CEILING = 1.910    # functions_NNPS.cuh:11


def initial_records(params, P1, k_table=None, l4=CASEH_L4, l_ceiling=CASEH_L_CEILING):
    """The reference's host pass over deck records before upload (in a copy)."""
    P = np.array(P1, dtype=PART1, copy=True)
    kt = None
    nk = 0
    if k_table is not None:
        z, k = k_table
        kt = np.ascontiguousarray(np.concatenate([np.asarray(z, np.float64), np.asarray(k, np.float64)]))
        nk = len(z)
    _check("sph_initial_records", lib().sph_initial_records(ctypes.byref(params), _p(P), len(P),
                                                            None if kt is None else _p(kt), nk,
                                                            float(l4), float(l_ceiling)))
    return P
