"""Reduced-precision storage against the FP64 oracle on a 128^3 crop of the
hall geometry (same cell size, materials and source as the 1024x768x512
hall), 4000 steps.  FP32 storage must match the FP32 oracle bit for bit and
the FP64 oracle to 1e-5 (relative L2 of the receiver IRs).  The 16-bit
storage errors are held to their measured values, and their 1e-3 target is
a strict expected failure."""
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


# Measured on this crop over 4000 steps on a B200 (round to nearest, the
# library's automatic storage scale; the GPU path equals the rounding
# oracle bit for bit): FP16 5.8e-3, BF16 2.4e-1.  The regression bound is
# 1.25x that; the 1e-3 target is a strict expected failure, so that a form
# meeting it shows up as an unexpected pass.
CROP_16BIT_MEASURED = {capi.STORAGE_F16: 5.8e-3, capi.STORAGE_BF16: 2.4e-1}
IR_TARGET = 1e-3


def _crop_16bit_error(crop, storage):
    sc, _, want64 = crop
    sim, _ = scenes.build_simulation(sc, storage=storage)
    sim.run(STEPS)
    got = sim.ir()
    sim.close()
    assert np.isfinite(got).all()
    err = rel_l2(got, want64)
    print(f"storage {storage}: IR rel-L2 vs FP64 = {err:.3e} over {STEPS} steps")
    return err


@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
def test_16bit_crop_error_regression(crop, storage):
    assert _crop_16bit_error(crop, storage) <= 1.25 * CROP_16BIT_MEASURED[storage]


@pytest.mark.xfail(strict=True, reason="16-bit storage on the hall crop: measured FP16 5.8e-3, BF16 2.4e-1 over "
                                       "4000 steps against the 1e-3 target")
@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
def test_16bit_crop_error_meets_target(crop, storage):
    assert _crop_16bit_error(crop, storage) <= IR_TARGET
