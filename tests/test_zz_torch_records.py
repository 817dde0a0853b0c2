"""Device-resident records from torch through the Python wrapper (needs a
B200).

Simulation.upload / download_into take CUDA arrays (__cuda_array_interface__)
as they are and hand their device pointers to the C ABI: a case uploaded
from a CUDA uint8 tensor steps exactly as the same records uploaded from
host memory, and its download into CUDA tensors holds the same bytes.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

pytestmark = pytest.mark.gpu


def test_torch_device_records_step_as_host_records():
    import torch
    P, p = decks.caseh_mini()
    n = len(P)
    host = abi.Simulation(p)
    host.upload(P)
    host.step(2)
    A1, A2, A3 = host.download()
    host.close()

    t_in = torch.from_numpy(P.view(np.uint8).copy()).cuda()
    outs = [torch.empty(n * dt.itemsize, dtype=torch.uint8, device="cuda")
            for dt in (layout.PART1, layout.PART2, layout.PART3)]
    torch.cuda.synchronize()
    sim = abi.Simulation(p)
    sim.upload(t_in)
    sim.step(2)
    sim.download_into(*outs)
    torch.cuda.synchronize()
    sim.close()
    for got, want in zip(outs, (A1, A2, A3)):
        assert got.cpu().numpy().tobytes() == want.tobytes()


def test_torch_device_array_of_the_wrong_size_is_refused():
    import torch
    P, p = decks.caseh_mini()
    sim = abi.Simulation(p)
    short = torch.empty((len(P) - 1) * layout.PART1.itemsize, dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError):
        sim.download_into(short)
    sim.close()
