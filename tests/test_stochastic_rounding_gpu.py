"""Stochastic rounding of the 16-bit stores (virs_set_rounding) against the
oracle, which defines the same rounding (oracle/virs_oracle.c, vo_sr16): the
random bits are a pure function of (voxel, step, phase), so the GPU path
must equal the oracle bit for bit, in every kernel variant, in batches and
in z-slabs (whose voxels take the whole grid's keys).

Accuracy on the 128^3 crop of the hall over 4000 steps against the FP64
oracle, as measured on a B200 (the library's automatic storage scale):
FP16 5.2e-3 (5.8e-3 to nearest), BF16 4.0e-2 (2.4e-1 to nearest).  Regression bound 1.25x that;
the 1e-3 target is a strict expected failure."""
import dataclasses

import numpy as np
import pytest

from helpers import oracle_grid, oracle_scene, rel_l2
from virs_b200 import capi, scenes, slabs

pytestmark = pytest.mark.gpu

SR = capi.ROUND_STOCHASTIC


def _scale(sc) -> float:
    peak = float(np.abs(sc.src_sig).max()) if sc.src_sig is not None and np.size(sc.src_sig) else 0.0
    if sc.hard is not None:
        peak = max(peak, float(np.abs(sc.hard).max()))
    return float(2.0 ** np.round(np.log2(1024.0 / peak))) if peak > 0 else 1.0


def _oracle_sr(sc, storage, scale):
    g = oracle_grid(sc)
    osc = oracle_scene(sc, g)
    osc.storage, osc.scale, osc.rounding = storage, scale, 1
    n = int(np.prod(g["shape"]))
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(g["bidx"].size * 12 + 1, np.float32))
    ir = osc.run(sc.steps, state=st)
    return ir, st[0]


def _fields_equal(sim, want_scaled, scale):
    p = sim.pressure().reshape(-1)
    want = want_scaled * np.float32(1.0 / scale)                  # unscaled on the GPU with flush-to-zero
    want[np.abs(want) < np.finfo(np.float32).tiny] *= np.float32(0.0)
    return np.array_equal(p.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
@pytest.mark.parametrize("depth", [0, 2])
def test_sr_matches_oracle_soft_source(storage, depth):
    """The 160x120x100 room (sponge 8, soft source): register and TMA kernels."""
    sc = scenes.plain_small(steps=400)
    scale = _scale(sc)
    want, want_p = _oracle_sr(sc, storage, scale)
    sim, _ = scenes.build_simulation(sc, storage=storage, storage_scale=scale)
    sim.set_rounding(SR)
    sim.set_tiling(8, 0, depth)
    sim.run(sc.steps)
    got = sim.ir()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), np.abs(got - want).max()
    assert _fields_equal(sim, want_p, scale)
    # the same run to nearest differs: the rounding is in effect
    near, _ = scenes.build_simulation(sc, storage=storage, storage_scale=scale)
    near.run(sc.steps)
    assert not np.array_equal(near.ir(), got)
    near.close()
    sim.close()


@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
def test_sr_matches_oracle_hard_source(storage):
    """The reference room: the speaker voxels' hard-source value (written by
    the post kernel with the step's key) and the reference boundary form."""
    sc = scenes.reference_room(steps=300)
    scale = _scale(dataclasses.replace(sc, hard=np.full(10, 10.0, np.float32)))
    want, want_p = _oracle_sr(sc, storage, scale)
    sim, _ = scenes.build_simulation(sc, storage=storage, storage_scale=scale)
    sim.set_rounding(SR)
    sim.run(sc.steps)
    got = sim.ir()
    assert np.abs(want).max() > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert _fields_equal(sim, want_p, scale)
    sim.close()


def test_sr_turns_two_steps_per_pass_off():
    """Two steps per pass do not apply stochastic rounding: asked for, they
    stay inactive and the run takes single steps, equal to the oracle."""
    sc = scenes.plain_small(steps=40)
    scale = _scale(sc)
    want, _ = _oracle_sr(sc, capi.STORAGE_BF16, scale)
    sim, _ = scenes.build_simulation(sc, storage=capi.STORAGE_BF16, storage_scale=scale)
    sim.set_rounding(SR)
    sim.set_time_blocking(2)
    assert not sim.time_blocking()["active"]
    sim.run(sc.steps)
    assert np.array_equal(sim.ir().view(np.uint32), want.view(np.uint32))
    sim.set_rounding(capi.ROUND_NEAREST)
    assert sim.time_blocking()["active"]
    sim.close()


def test_sr_batch_members_equal_solo_runs():
    scs = scenes.batched(steps=70, n_sources=2, n_rooms=2, room=64, size_range=(40, 80))
    alone = []
    for sc in scs:
        sim, _ = scenes.build_simulation(sc, storage=capi.STORAGE_BF16)
        sim.set_rounding(SR)
        sim.run(sc.steps)
        alone.append(sim.ir())
        sim.close()
    sims = []
    for sc in scs:
        s, _ = scenes.build_simulation(sc, storage=capi.STORAGE_BF16)
        s.set_rounding(SR)
        sims.append(s)
    with capi.Batch(sims) as b:
        b.run(70)
        b.synchronize()
        for sim, want in zip(sims, alone):
            assert np.array_equal(sim.ir().view(np.uint32), want.view(np.uint32))
    for s in sims:
        s.close()


def test_sr_slabs_equal_whole_grid():
    """Two slabs on one GPU: their voxels take the whole grid's keys."""
    import torch
    sc = dataclasses.replace(scenes.furnished_room(steps=120), cell_size=1 / 32, sponge_width=6)
    scale = 64.0
    whole, _ = scenes.build_simulation(sc, storage=capi.STORAGE_BF16, storage_scale=scale)
    whole.set_rounding(SR)
    parts, _ = scenes.build_slabs(sc, 2, storage=capi.STORAGE_BF16, storage_scale=scale)
    for s, *_ in parts:
        s.set_rounding(SR)
    whole.run(sc.steps)
    want_ir = whole.ir()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(sc.steps):
        slabs.exchange_local([p[0] for p in parts])
        for s, *_ in parts:
            s.run(1, stream=stream)
    torch.cuda.synchronize()
    ir = np.zeros_like(want_ir)
    for s, _, _, own_r in parts:
        if own_r.any():
            ir[own_r] = s.ir()
    assert np.abs(want_ir).max() > 0
    assert np.array_equal(ir.view(np.uint32), want_ir.view(np.uint32))
    for s, *_ in parts:
        s.close()
    whole.close()


# ---- accuracy against FP64 on the hall crop -------------------------------------

STEPS = 4000
CROP_SR_MEASURED = {capi.STORAGE_F16: 5.2e-3, capi.STORAGE_BF16: 4.0e-2}
IR_TARGET = 1e-3


@pytest.fixture(scope="module")
def crop():
    sc = scenes.large_hall(steps=STEPS, size=(128, 128, 128))
    g = oracle_grid(sc)
    return sc, oracle_scene(sc, g).run(STEPS, f64=True)


def _crop_sr_error(crop, storage):
    sc, want64 = crop
    sim, _ = scenes.build_simulation(sc, storage=storage)
    sim.set_rounding(SR)
    sim.run(STEPS)
    got = sim.ir()
    sim.close()
    assert np.isfinite(got).all()
    err = rel_l2(got, want64)
    print(f"storage {storage}, stochastic rounding: IR rel-L2 vs FP64 = {err:.3e} over {STEPS} steps")
    return err


@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
def test_sr_crop_error_regression(crop, storage):
    assert _crop_sr_error(crop, storage) <= 1.25 * CROP_SR_MEASURED[storage]


@pytest.mark.xfail(strict=True, reason="stochastic rounding on the hall crop: measured FP16 5.2e-3, BF16 4.0e-2 "
                                       "over 4000 steps against the 1e-3 target")
@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
def test_sr_crop_error_meets_target(crop, storage):
    assert _crop_sr_error(crop, storage) <= IR_TARGET
