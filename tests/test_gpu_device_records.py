"""Records in device memory through the C ABI (needs a B200).

The reference keeps its records on the device (dev_P1, dev_P2 of
ISPH_Calc.cuh:327-344), so sph_upload and sph_download also take device
pointers.  A case uploaded from device memory steps exactly as the same case
uploaded from host memory, its downloads into device memory hold the same
bytes, and the property-table check of a step sees the records' p_type
classes wherever they were uploaded from.
"""
import ctypes

import numpy as np
import pytest

from sph_b200 import abi, decks, layout

pytestmark = pytest.mark.gpu

H2D, D2H = 1, 2


def _cudart():
    abi.lib()   # the library's own runtime, already loaded by soname
    L = ctypes.CDLL("libcudart.so.12")
    L.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
    L.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    L.cudaFree.argtypes = [ctypes.c_void_p]
    return L


class DeviceBuffer:
    def __init__(self, nbytes):
        self.L = _cudart()
        self.ptr = ctypes.c_void_p()
        assert self.L.cudaMalloc(ctypes.byref(self.ptr), nbytes) == 0
        self.nbytes = nbytes

    def put(self, arr):
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes == self.nbytes
        assert self.L.cudaMemcpy(self.ptr, arr.ctypes.data, self.nbytes, H2D) == 0

    def get(self, dtype):
        out = np.zeros(self.nbytes // np.dtype(dtype).itemsize, dtype)
        assert self.L.cudaMemcpy(out.ctypes.data, self.ptr, self.nbytes, D2H) == 0
        return out

    def free(self):
        self.L.cudaFree(self.ptr)


def test_device_records_step_as_host_records():
    P, p = decks.caseh_mini()
    n = len(P)
    host = abi.Simulation(p)
    host.upload(P)
    host.step(2)
    A1, A2, A3 = host.download()
    host.close()

    d_in = DeviceBuffer(n * layout.PART1.itemsize)
    d_in.put(P)
    outs = [DeviceBuffer(n * dt.itemsize) for dt in (layout.PART1, layout.PART2, layout.PART3)]
    sim = abi.Simulation(p)
    L = abi.lib()
    assert L.sph_upload(sim.h, d_in.ptr, None, n) == 0
    sim.step(2)
    assert L.sph_download(sim.h, outs[0].ptr, outs[1].ptr, outs[2].ptr) == 0
    B1, B2, B3 = (b.get(dt) for b, dt in zip(outs, (layout.PART1, layout.PART2, layout.PART3)))
    # and a host download of the same context
    C1, _, _ = sim.download()
    sim.close()
    for b in [d_in] + outs:
        b.free()
    assert B1.tobytes() == A1.tobytes()
    assert B2.tobytes() == A2.tobytes()
    assert B3.tobytes() == A3.tobytes()
    assert C1.tobytes() == A1.tobytes()


def test_table_check_sees_device_records():
    P, p, tables = decks.enthalpy_tables_mini()
    q = p.copy()
    q.ppe_mode = layout.PPE_REF_SWEEP
    L = abi.lib()
    # a served deck steps
    d = DeviceBuffer(len(P) * layout.PART1.itemsize)
    d.put(P)
    sim = abi.Simulation(q)
    sim.set_prop_tables(tables)
    assert L.sph_upload(sim.h, d.ptr, None, len(P)) == 0
    sim.step(1)
    sim.close()
    # one fluid record with |p_type| 12, which no table serves: refused
    Q = P.copy()
    k = int(np.nonzero((Q["p_type"] == 1) & (Q["i_type"] < 3))[0][0])
    Q["p_type"][k] = -12
    d.put(Q)
    sim = abi.Simulation(q)
    sim.set_prop_tables(tables)
    assert L.sph_upload(sim.h, d.ptr, None, len(Q)) == 0
    with pytest.raises(abi.SphError):
        sim.step(1)
    sim.close()
    d.free()
