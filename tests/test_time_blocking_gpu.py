"""Two steps per pass (virs_set_time_blocking) against the oracle and
against single steps, bit for bit.

The two-step kernel computes p^{n+2} before the first step's boundary pass
and post kernel have run; the voxels next to boundary voxels and sources are
recomputed afterwards.  These cases put walls, boundary voxels, hard and
soft sources and receivers next to tile edges, z-chunk edges and the grid
border, on sizes that are not multiples of the tiles, in FP32 and in 16-bit
storage, through CUDA graphs, eager launches, timed launches and the single
steps that finish a run whose length is not a multiple of four.
"""
import numpy as np
import pytest

import oracle
from helpers import oracle_grid, oracle_scene
from virs_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def _random_case(shape, W, seed, steps):
    """Scattered walls (flag 1) and hard sources (flag 3), 3 materials x 2
    sections, 3 soft sources and 4 receivers; the oracle's receiver samples
    and final fields."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    n = nx * ny * nz
    flags = np.zeros(n, np.uint8)
    flags[rng.random(n) < 0.03] = 1
    flags[rng.random(n) < 0.001] = 3
    wmat = rng.integers(0, 3, n).astype(np.uint8)
    ref_flags, bmat_full, bd2_full = oracle.classify(shape, W, flags, wmat)
    bidx = oracle.boundary_list(shape, ref_flags)
    coef = np.stack([capi.design_octave_cascade(40000.0, a)[:2] for a in rng.uniform(0.1, 0.7, (3, 3))])
    air = np.flatnonzero((ref_flags == 0) | (ref_flags == 2))
    xs, ys, zs = air % nx, (air // nx) % ny, air // (nx * ny)
    inner = air[(xs > 0) & (ys > 0) & (zs > 0) & (xs < nx - 1) & (ys < ny - 1) & (zs < nz - 1)]
    src = rng.choice(inner, 3, replace=False).astype(np.uint64)
    rcv = rng.choice(inner, 4, replace=False).astype(np.uint64)
    sig = rng.standard_normal((3, 80)).astype(np.float32)
    hard = rng.uniform(-2, 2, 50).astype(np.float32)

    def make():
        sim = capi.Simulation(capi.default_params(sponge_width=W, courant=1.0, boundary_form=1))
        sim.set_grid(shape, 0.05, flags, wmat)
        sim.classify()
        sim.set_filters(coef.astype(np.float32), n_sections=2)
        sim.set_sources(src, sig)
        sim.set_receivers(rcv)
        sim.set_hard_source(hard)
        sim.start(steps)
        return sim

    _, c2dt2, inv_h2, K = oracle.step_constants(0.05, 343.0, 1.0)
    osc = oracle.Scene(shape, ref_flags, bidx, bmat_full[bidx], oracle.sponge_weights_for(W, bd2_full[bidx]),
                       coef.astype(np.float32), 2, hard=hard, src_idx=src, src_sig=sig, rcv_idx=rcv,
                       consts=(c2dt2, inv_h2, K), form=1)
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(bidx.size * 8 + 1, np.float32))
    want = osc.run(steps, state=st)
    return make, want, st


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.mark.parametrize("shape,W,seed,rows,planes", [
    ((37, 29, 23), 1, 0, 16, 0),
    ((130, 17, 21), 3, 2, 32, 5),
    ((300, 40, 30), 2, 5, 16, 7),
    ((33, 64, 40), 5, 3, 32, 0),
    ((250, 31, 18), 1, 6, 16, 1),
    ((45, 27, 19), 2, 7, 14, 3),
    ((270, 23, 25), 1, 8, 12, 0),
    ((64, 50, 30), 3, 9, 12, 6),
])
def test_random_grids_match_oracle(shape, W, seed, rows, planes):
    """123 steps: 30 groups of four (a CUDA graph of eight, then eager
    launches) and three single steps."""
    steps = 123
    make, want, st = _random_case(shape, W, seed, steps)
    sim = make()
    sim.set_time_blocking(2, rows, planes)
    assert sim.time_blocking()["active"]
    sim.run(steps)
    assert np.abs(want).max() > 0
    assert _same(sim.ir(), want)
    p, pp = sim.pressure(prev=True)
    assert _same(p.reshape(-1), st[0])
    assert _same(pp.reshape(-1), st[1])
    sim.close()


def test_run_lengths_timing_and_single_steps_agree():
    """Runs of 5, 7, 40 and 3 steps (groups of four and leftovers), timed and
    untimed, give the samples and fields of single steps."""
    shape, steps = (70, 45, 33), 55
    make, want, st = _random_case(shape, 2, 11, steps)
    a = make()
    a.run(steps)
    base, (bp, bpp) = a.ir(), a.pressure(prev=True)
    assert _same(base, want)
    a.close()
    for timed in (False, True):
        b = make()
        b.set_time_blocking(2)
        if timed:
            b.set_timing(True)
        for k in (5, 7, 40, 3):
            b.run(k)
        assert _same(b.ir(), base)
        p, pp = b.pressure(prev=True)
        assert _same(p, bp) and _same(pp, bpp)
        if timed:
            t = b.timing()
            # 5 = 4 + 1, 7 = 4 + 3, 40 = 10 x 4, 3: 12 groups of four are 24
            # two-step launches, plus 7 single steps
            assert t.step_launches == 24 + 7
            assert t.step_kernel_ms > 0
        b.close()


@pytest.mark.parametrize("storage", [capi.STORAGE_F32, capi.STORAGE_BF16, capi.STORAGE_F16])
def test_wide_hall_matches_oracle(storage):
    """A hall three tiles wide with a floor material, FP32 and 16-bit
    storage (rounded like the oracle's storage run)."""
    sc = scenes.large_hall(steps=202, size=(384, 80, 72))
    g = oracle_grid(sc)
    osc = oracle_scene(sc, g)
    scale = 1.0
    if storage != capi.STORAGE_F32:
        peak = float(np.abs(sc.src_sig).max())
        scale = float(2.0 ** np.round(np.log2(1024.0 / peak)))
        osc.storage, osc.scale = storage, scale
    n = int(np.prod(g["shape"]))
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(g["bidx"].size * 12 + 1, np.float32))
    want = osc.run(sc.steps, state=st)
    sim, _ = scenes.build_simulation(sc, storage=storage, storage_scale=scale if storage else 0.0)
    sim.set_time_blocking(2, 16, 0)
    sim.run(sc.steps)
    assert np.abs(want).max() > 0
    assert _same(sim.ir(), want), np.abs(sim.ir() - want).max()
    p = sim.pressure().reshape(-1)
    want_p = st[0] * np.float32(1.0 / scale)
    if storage != capi.STORAGE_F32:
        want_p[np.abs(want_p) < np.finfo(np.float32).tiny] *= np.float32(0.0)
    assert _same(p, want_p)
    sim.close()


def test_moved_sources_rebuild_the_fix_list():
    """Sources moved between runs: the voxels around the new positions are
    recomputed, so the run still equals single steps."""
    shape, steps = (64, 40, 36), 48
    make, _, _ = _random_case(shape, 1, 21, steps)
    nx, ny, _ = shape
    runs = []
    for pair in (False, True):
        s = make()
        if pair:
            s.set_time_blocking(2)
        s.run(steps)
        flags = s.flags()
        inner = np.flatnonzero(flags.reshape(-1) == 0)
        x, y, z = inner % nx, (inner // nx) % ny, inner // (nx * ny)
        inner = inner[(x > 2) & (y > 2) & (z > 2) & (x < nx - 3) & (y < ny - 3)]
        src = inner[[5, len(inner) // 2]].astype(np.uint64)
        s.set_sources(src, np.ones((2, 30), np.float32))
        s.start(steps)
        s.run(steps)
        runs.append((s.ir(), s.pressure()))
        s.close()
    assert _same(runs[0][0], runs[1][0]) and _same(runs[0][1], runs[1][1])


@pytest.mark.parametrize("lead", [0, 1, 2, 3])
def test_stop_rule_inside_a_group_of_four(lead):
    """The device stop rule fires at the same step as with single steps,
    wherever that step falls in a group of four (lead single steps shift the
    groups), and leaves the same samples and fields."""
    sc = scenes.reference_room(steps=3200, size=(24, 20, 16))
    ref, _ = scenes.build_simulation(sc)
    ref.set_stop_rule(True)
    ref.run(sc.steps)
    stopped, stop = ref.stop_state()
    assert stopped and stop > 3000
    dev, _ = scenes.build_simulation(sc)
    dev.set_stop_rule(True)
    dev.set_time_blocking(2)
    assert dev.time_blocking()["active"]
    if lead:
        dev.run(lead)
    dev.run(sc.steps - lead)
    assert dev.stop_state() == (True, stop)
    assert dev.info().steps_done == stop + 1
    assert _same(dev.ir(0, stop + 1), ref.ir(0, stop + 1))
    p, pp = dev.pressure(prev=True)
    rp, rpp = ref.pressure(prev=True)
    assert _same(p, rp) and _same(pp, rpp)
    dev.run(8)                                              # nothing runs after the stop
    assert dev.info().steps_done == stop + 1
    assert _same(dev.pressure(), rp)
    ref.close()
    dev.close()


def test_not_used_with_the_register_kernel():
    make, want, _ = _random_case((40, 30, 20), 1, 3, 20)
    sim = make()
    sim.set_time_blocking(2)
    assert sim.time_blocking()["active"]
    sim.set_stop_rule(True)
    assert sim.time_blocking()["active"]
    sim.set_stop_rule(False)
    sim.set_tiling(8, 0, 0)
    assert not sim.time_blocking()["active"]
    sim.run(20)
    assert _same(sim.ir(), want)
    sim.set_tiling(8, 0, 2)
    assert sim.time_blocking()["active"]
    sim.set_time_blocking(1)
    assert sim.time_blocking() == {"steps_per_pass": 1, "rows": 14, "planes": 0, "active": False}
    with pytest.raises(capi.VirsError):
        sim.set_time_blocking(3)
    with pytest.raises(capi.VirsError):
        sim.set_time_blocking(2, 8)
    sim.close()


def test_adjoint_forward_pass_and_gradients_unchanged():
    """virs_forward_checkpointed advances its segments through virs_run, so
    with two steps per pass: the same receiver samples bit for bit, and the
    same gradients (their FP64 sums are accumulated with atomics, whose order
    varies from run to run, so they agree to 1e-9 relative)."""
    sc, _ = scenes.inverse_design(steps=200, size=(40, 36, 28), h=0.04, n_materials=6)
    dl = np.random.default_rng(5).standard_normal((len(sc.rcv_pos), sc.steps)).astype(np.float32)
    out = []
    for pair in (False, True):
        sim, _ = scenes.build_simulation(sc)
        if pair:
            sim.set_time_blocking(2)
            assert sim.time_blocking()["active"]
        sim.forward_checkpointed(sc.steps, 32)
        ir = sim.ir(0, sc.steps)
        gc, gs = sim.adjoint(dl, sc.n_materials, sc.n_sections)
        out.append((ir, gc, gs))
        sim.close()
    assert _same(out[0][0], out[1][0])
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max()


def test_batch_of_members_that_ran_two_steps_per_pass():
    """Members advanced two steps per pass keep their state in the usual two
    buffers, so a batch built from them continues exactly as their solo
    runs."""
    shape, steps = (64, 40, 36), 48
    solo = []
    for seed in (31, 32):
        make, _, _ = _random_case(shape, 1, seed, steps)
        s = make()
        s.run(steps)
        solo.append(s.ir())
        s.close()
    members = []
    for seed in (31, 32):
        make, _, _ = _random_case(shape, 1, seed, steps)
        s = make()
        s.set_time_blocking(2)
        s.run(20)                                   # five groups of four
        members.append(s)
    batch = capi.Batch(members)
    batch.run(steps - 20)
    batch.synchronize()
    for m, want in zip(members, solo):
        assert _same(m.ir(), want)
    batch.close()
    for m in members:
        m.close()


@pytest.mark.parametrize("shape", [(3, 3, 3), (5, 4, 3), (33, 3, 7), (130, 5, 4), (260, 17, 9), (40, 40, 5)])
def test_degenerate_grids(shape):
    """One interior voxel, one interior plane, grids thinner than a tile in
    y, narrower than a tile in x and wider than two: two steps per pass
    equal the oracle."""
    nx, ny, nz = shape
    n = nx * ny * nz
    rng = np.random.default_rng(sum(shape))
    flags = np.zeros(n, np.uint8)
    if n > 27:
        flags[rng.random(n) < 0.05] = 1
    ref_flags, bm, bd = oracle.classify(shape, 1, flags, None)
    bidx = oracle.boundary_list(shape, ref_flags)
    interior = [i for i in range(n)
                if 0 < i % nx < nx - 1 and 0 < (i // nx) % ny < ny - 1 and 0 < i // (nx * ny) < nz - 1
                and ref_flags[i] in (0, 2)]
    src = np.array(interior[:1], np.uint64)
    rcv = np.array(interior[-2:], np.uint64)
    sig = np.linspace(-1, 1, 30, dtype=np.float32)[None, :]
    steps = 26
    _, c2dt2, inv_h2, K = oracle.step_constants(0.05, 343.0, 1.0)
    fs = oracle.filter_fs(0.05, 343.0, 1.0)
    coef = oracle.rbj_highpass_ref(fs, 440.0, 0.1)[None, None, :]
    osc = oracle.Scene(shape, ref_flags, bidx, bm[bidx], oracle.sponge_weights_for(1, bd[bidx]), coef, 1,
                       hard=np.full(10, 10.0, np.float32), src_idx=src, src_sig=sig, rcv_idx=rcv,
                       consts=(c2dt2, inv_h2, K), form=1)
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(bidx.size * 4 + 1, np.float32))
    want = osc.run(steps, state=st)
    sim = capi.Simulation(capi.default_params(courant=1.0, boundary_form=1))
    sim.set_grid(shape, 0.05, flags)
    sim.classify()
    sim.set_sources(src, sig)
    sim.set_receivers(rcv)
    sim.start(steps)
    sim.set_time_blocking(2, 16, 0)
    assert sim.time_blocking()["active"]
    sim.run(steps)
    assert _same(sim.ir(), want)
    p, pp = sim.pressure(prev=True)
    assert _same(p, st[0]) and _same(pp, st[1])
    sim.close()
