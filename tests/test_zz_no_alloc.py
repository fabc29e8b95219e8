"""virs_energy_noalloc: the energy monitor for callers that cannot allocate
device memory (real-time threads, where cudaMalloc/cudaFree may block on a
device-wide synchronisation, or hosts that own all device memory through a
pool).  Its scratch is a static device array instead of a buffer allocated
on first use, so it is checked against virs_energy, which allocates.

Kept in a file of its own that pytest collects last: a run that stops at
the first failure has then already run every other test."""
import numpy as np
import pytest

from virs_b200 import capi, scenes

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9      # the tolerance of the other energy-monitor checks


@pytest.mark.parametrize("storage", [capi.STORAGE_F32, capi.STORAGE_BF16, capi.STORAGE_F16])
def test_energy_noalloc_matches_energy_on_two_calls(storage):
    """FP32, BF16 and FP16 fields: each storage type has its own conversion
    and the inverse scale squared in the sum."""
    import torch
    sc = scenes.plain_small(steps=300)
    sim, _ = scenes.build_simulation(sc, storage=storage)
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")   # the caller's output buffer
    side = torch.cuda.Stream()
    for k in range(2):
        sim.run(150)
        want = sim.energy()
        if k == 0:
            sim.energy_noalloc(out[0:1].data_ptr())                   # the handle's own stream
            sim.synchronize()
        else:
            sim.energy_noalloc(out[1:2].data_ptr(), side.cuda_stream)  # a caller's stream
            side.synchronize()
        got = float(out[k].item())
        assert want > 0
        assert abs(got - want) <= REL_TOL * abs(want), (k, got, want)
    sim.close()                                                   # waits for the reads on `side` too


def test_energy_noalloc_rejects_grids_beyond_the_scratch():
    import torch
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    nz = 8193                                                     # VIRS_ENERGY_MAX_PLANES + 1
    shape = (3, 3, nz)
    sim = capi.Simulation()
    sim.set_grid(shape, 0.05, np.zeros(9 * nz, np.uint8))
    sim.classify()
    with pytest.raises(capi.VirsError) as e:
        sim.energy_noalloc(out.data_ptr())
    assert e.value.status == capi.E_ARG
    assert "8192" in str(e.value)
    sim.close()
