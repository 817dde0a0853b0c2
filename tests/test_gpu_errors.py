"""Error behaviour of the C ABI on a GPU (needs a B200): calls out of order
and bad arguments return the documented status and leave the context usable;
no call aborts the process."""
import ctypes

import numpy as np
import pytest

from sph_b200 import abi, decks, layout

pytestmark = pytest.mark.gpu

BAD_ARG, STATE = -1, -4


def _ctx():
    P, p = decks.caseh_mini(nx=8, ny=4, nz=4)
    return P, p, abi.Simulation(p, precision=layout.PREC_MIXED)


def test_calls_before_upload_report_state_errors():
    P, p, sim = _ctx()
    L = abi.lib()
    st = abi.PpeStats()
    assert L.sph_step(sim.h, 1, ctypes.byref(st)) == STATE
    assert L.sph_nnps(sim.h) == STATE
    g = np.zeros(len(P), np.int32)
    assert L.sph_nnps_export(sim.h, g.ctypes.data_as(ctypes.c_void_p), None, None, None) == STATE
    assert b"uploaded" in L.sph_last_error() or b"NNPS" in L.sph_last_error()
    # the context still works after the errors
    sim.upload(P)
    s = sim.step(1)
    assert s.status in (0, 1)
    sim.close()


def test_wrong_particle_count_is_rejected():
    P, p, sim = _ctx()
    L = abi.lib()
    Q = np.ascontiguousarray(P[:-1])
    assert L.sph_upload(sim.h, Q.ctypes.data_as(ctypes.c_void_p), None, len(Q)) == BAD_ARG
    assert b"num_part2" in L.sph_last_error()
    sim.upload(P)
    sim.step(1)
    sim.close()


def test_params_that_change_the_grid_are_rejected():
    P, p, sim = _ctx()
    sim.upload(P)
    q = p.copy()
    q.seti("num_cells", p.geti("num_cells") + 7)
    with pytest.raises(abi.SphError) as e:
        sim.set_params(q)
    assert e.value.status == BAD_ARG
    sim.close()
