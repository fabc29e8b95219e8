"""Reduced-precision storage against the FP64 oracle on a 128^3 crop of the
hall geometry (same cell size, materials and source as the 1024x768x512
hall), 4000 steps.  FP32 storage must match the FP32 oracle bit for bit and
the FP64 oracle to 1e-5 (relative L2 of the receiver IRs); the 16-bit
storage errors are measured and bounded."""
import numpy as np
import pytest

from helpers import oracle_grid, oracle_scene, rel_l2
from virs_b200 import capi, scenes

pytestmark = pytest.mark.gpu

STEPS = 4000


@pytest.fixture(scope="module")
def crop():
    sc = scenes.large_hall(steps=STEPS, size=(128, 128, 128))
    g = oracle_grid(sc)
    osc = oracle_scene(sc, g)
    return sc, osc.run(STEPS), osc.run(STEPS, f64=True)


def test_fp32_crop_matches_oracles(crop):
    sc, want32, want64 = crop
    sim, _ = scenes.build_simulation(sc)
    sim.run(STEPS)
    got = sim.ir()
    assert np.array_equal(got.view(np.uint32), want32.view(np.uint32))
    err = rel_l2(got, want64)
    print(f"FP32 storage: IR rel-L2 vs FP64 = {err:.3e}")
    assert err <= 1e-5
    sim.close()


@pytest.mark.parametrize("storage,bound", [(capi.STORAGE_F16, 5e-2), (capi.STORAGE_BF16, 3e-1)])
def test_16bit_crop_error(crop, storage, bound):
    sc, _, want64 = crop
    sim, _ = scenes.build_simulation(sc, storage=storage)
    sim.run(STEPS)
    got = sim.ir()
    err = rel_l2(got, want64)
    print(f"storage {storage}: IR rel-L2 vs FP64 = {err:.3e} over {STEPS} steps")
    assert np.isfinite(got).all() and err <= bound
    sim.close()
