"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Integer work (flags, normals, boundary lists, materials) must match bit for
bit.  The FP32 step uses the same operation order as the oracle (explicit
fused multiply-adds, flush-to-zero, the double-precision boundary
correction), so receiver samples and fields must match bit for bit too; the
relative-L2 bound of 1e-5 against the FP64 oracle is checked on top.
"""
import dataclasses

import numpy as np
import pytest

import oracle
from helpers import grid_parity, oracle_grid, oracle_scene, rel_l2
from virs_b200 import capi, scenes

pytestmark = pytest.mark.gpu

FP32_REL_L2 = 1e-5


_grid_parity = grid_parity


def test_reference_room_bit_exact():
    sc = scenes.reference_room(steps=300)
    g = oracle_grid(sc)
    sim, meta = scenes.build_simulation(sc)
    _grid_parity(sim, g)
    osc = oracle_scene(sc, g)
    st = (np.zeros(int(np.prod(g["shape"])), np.float32), np.zeros(int(np.prod(g["shape"])), np.float32),
          np.zeros(g["bidx"].size * 4 + 1, np.float32))
    want = osc.run(sc.steps, state=st)
    sim.run(sc.steps)
    got = sim.ir()
    assert np.abs(want).max() > 1e-3
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    p, pp = sim.pressure(prev=True)
    assert np.array_equal(p.view(np.uint32), st[0].view(np.uint32))
    assert np.array_equal(pp.view(np.uint32), st[1].view(np.uint32))
    sim.close()


def test_plain_small_config_bit_exact():
    """160x120x100, 6 first-order absorbers, sponge 8, Courant 1/sqrt 3."""
    sc = scenes.plain_small(steps=2000)
    g = oracle_grid(sc)
    sim, meta = scenes.build_simulation(sc)
    _grid_parity(sim, g)
    assert set(np.unique(g["bmat"]).tolist()) == set(range(6))
    osc = oracle_scene(sc, g)
    want = osc.run(sc.steps)
    sim.run(sc.steps)
    got = sim.ir()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    want64 = osc.run(sc.steps, f64=True)
    assert rel_l2(got, want64) <= FP32_REL_L2
    sim.close()


def test_furnished_room_reduced_bit_exact():
    """The furnished-room generator (boxes, 4 materials, 3-section cascades)
    at half resolution and sponge 6, 600 steps."""
    sc = scenes.furnished_room(steps=600)
    sc = dataclasses.replace(sc, cell_size=1 / 32, sponge_width=6)
    g = oracle_grid(sc)
    sim, meta = scenes.build_simulation(sc)
    _grid_parity(sim, g)
    osc = oracle_scene(sc, g)
    want = osc.run(sc.steps)
    sim.run(sc.steps)
    got = sim.ir()
    assert got.shape == (4, sc.steps)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    sim.close()


@pytest.mark.parametrize("shape,W,seed", [((37, 29, 23), 1, 0), ((70, 33, 19), 2, 1), ((130, 17, 21), 3, 2),
                                          ((33, 64, 40), 5, 3), ((48, 48, 48), 16, 4)])
def test_random_grids_bit_exact(shape, W, seed):
    """Scattered walls (flag 1) and hard sources (flag 3) on odd-sized grids;
    sizes that are not multiples of the row padding or of the tiles."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    n = nx * ny * nz
    flags = np.zeros(n, np.uint8)
    flags[rng.random(n) < 0.03] = 1
    flags[rng.random(n) < 0.001] = 3
    wmat = rng.integers(0, 3, n).astype(np.uint8)
    ref_flags, bmat_full, bd2_full = oracle.classify(shape, W, flags, wmat)
    bidx = oracle.boundary_list(shape, ref_flags)
    p = capi.default_params(sponge_width=W, courant=1.0, boundary_form=1)
    sim = capi.Simulation(p)
    sim.set_grid(shape, 0.05, flags, wmat)
    sim.classify()
    assert np.array_equal(sim.flags(), ref_flags)
    assert np.array_equal(sim.normals(), oracle.normals(shape, ref_flags))
    assert np.array_equal(sim.boundary_indices(), bidx)
    m, w = sim.boundary_materials()
    assert np.array_equal(m, bmat_full[bidx])
    assert np.array_equal(w, oracle.sponge_weights_for(W, bd2_full[bidx]))
    # a short run with 3 materials x 2 sections, soft sources and receivers
    coef = np.stack([capi.design_octave_cascade(40000.0, a)[:2] for a in rng.uniform(0.1, 0.7, (3, 3))])
    sim.set_filters(coef.astype(np.float32), n_sections=2)
    air = np.flatnonzero((ref_flags == 0) | (ref_flags == 2))
    xs, ys, zs = air % nx, (air // nx) % ny, air // (nx * ny)
    inner = air[(xs > 0) & (ys > 0) & (zs > 0) & (xs < nx - 1) & (ys < ny - 1) & (zs < nz - 1)]
    src = rng.choice(inner, 3, replace=False).astype(np.uint64)
    rcv = rng.choice(inner, 4, replace=False).astype(np.uint64)
    sig = rng.standard_normal((3, 80)).astype(np.float32)
    hard = rng.uniform(-2, 2, 50).astype(np.float32)
    sim.set_sources(src, sig)
    sim.set_receivers(rcv)
    sim.set_hard_source(hard)
    steps = 120
    sim.start(steps)
    sim.run(steps)
    dt, c2dt2, inv_h2, K = oracle.step_constants(0.05, 343.0, 1.0)
    osc = oracle.Scene(shape, ref_flags, bidx, bmat_full[bidx], oracle.sponge_weights_for(W, bd2_full[bidx]),
                       coef.astype(np.float32), 2, hard=hard, src_idx=src, src_sig=sig, rcv_idx=rcv,
                       consts=(c2dt2, inv_h2, K), form=1)
    N = n
    st = (np.zeros(N, np.float32), np.zeros(N, np.float32), np.zeros(bidx.size * 8 + 1, np.float32))
    want = osc.run(steps, state=st)
    assert np.array_equal(sim.ir().view(np.uint32), want.view(np.uint32))
    p = sim.pressure()
    assert np.array_equal(p.view(np.uint32), st[0].view(np.uint32))
    sim.close()


@pytest.mark.parametrize("rows,planes,depth", [(4, 1, 0), (8, 7, 1), (16, 32, 2), (8, 0, 3), (4, 500, 2),
                                               (16, 3, 0), (8, 0, 0)])
def test_tilings_agree(rows, planes, depth):
    """Every kernel variant (register streaming, TMA at depth 1..3) and tiling
    gives the same bits as the default."""
    sc = scenes.plain_small(steps=150)
    sim, _ = scenes.build_simulation(sc)
    sim.run(sc.steps)
    base = sim.ir()
    pbase = sim.pressure()
    sim.set_tiling(rows, planes, depth)
    sim.start(sc.steps)
    sim.run(sc.steps)
    assert np.array_equal(sim.ir().view(np.uint32), base.view(np.uint32))
    assert np.array_equal(sim.pressure().view(np.uint32), pbase.view(np.uint32))
    sim.close()


def test_graph_steps_and_host_runs_agree():
    """virs_run (CUDA graph chunks + remainder), virs_step (one launch per
    step) and virs_run_host (host buffers) give the same samples."""
    sc = scenes.reference_room(steps=101)
    a, _ = scenes.build_simulation(sc)
    a.run(sc.steps)
    ir_graph = a.ir()
    a.start(sc.steps)
    for n in range(sc.steps):
        keep, v = a.step(n)
        assert keep
        assert v == ir_graph[0, n]
    assert np.array_equal(a.ir(), ir_graph)
    a.start(sc.steps)
    out = np.zeros((3, 60), np.float32)
    a.run_host(60, None, out)
    out2 = np.zeros((3, 41), np.float32)
    a.run_host(41, None, out2)
    assert np.array_equal(np.concatenate([out, out2], 1), ir_graph)
    a.close()


def test_run_host_signal_chunks():
    sc = scenes.plain_small(steps=200)
    a, meta = scenes.build_simulation(sc)
    a.run(sc.steps)
    want = a.ir()
    a.start(sc.steps)
    ir = np.zeros((1, 100), np.float32)
    a.run_host(100, sc.src_sig[:, :100].copy(), ir)
    ir2 = np.zeros((1, 100), np.float32)
    a.run_host(100, sc.src_sig[:, 100:].copy(), ir2)
    assert np.array_equal(np.concatenate([ir, ir2], 1), want)
    a.close()


def test_rms_stop_rule():
    """virs_step's stop decision follows simulator_gpu.cu:303-330."""
    sc = scenes.reference_room(steps=3200, size=(24, 20, 16))
    sim, _ = scenes.build_simulation(sc)
    keep = []
    for n in range(sc.steps):
        k, _ = sim.step(n)
        keep.append(k)
    out = sim.ir()[0]
    state = 0.0
    want = []
    for step in range(sc.steps):
        go = True
        if step > 3000:
            s = np.float32(0)
            for i in range(step - 100, step):
                s = np.float32(s + np.float32(out[i] * out[i]))
            rms = np.float32(np.sqrt(np.float32(s / np.float32(100))))
            if step == 3001:
                state = rms
            else:
                g = np.float32(8e-5)
                vout = np.float32(np.float32(g * rms + state) / np.float32(g + 1))
                state = np.float32(2 * vout - state)
                rms = vout
            go = not (rms < np.float32(0.0009))
        want.append(go)
    assert keep == want
    sim.close()


def test_energy_monitor_matches_oracle_and_is_conserved():
    shape = (40, 36, 30)
    nx, ny, nz = shape
    f = np.zeros((nz, ny, nx), np.uint8)
    f[0], f[-1], f[:, 0], f[:, -1], f[:, :, 0], f[:, :, -1] = 1, 1, 1, 1, 1, 1
    f = f.reshape(-1)
    p = capi.default_params(boundary_gain=0.0, courant=1.0)
    sim = capi.Simulation(p)
    sim.set_grid(shape, 0.05, f)
    sim.classify()
    sim.set_receivers([((15 * ny) + 18) * nx + 20])
    sim.start(400)
    sim.init_pressure_sphere(20, 18, 15, 4, 1.0, True)
    e0 = sim.energy()
    cur, prev = sim.pressure(prev=True)
    ref_flags, _, _ = oracle.classify(shape, 1, f)
    dt, c2dt2, inv_h2, K = oracle.step_constants(0.05, 343.0, 1.0)
    e_or = oracle.energy(shape, ref_flags, cur, prev, float(c2dt2) * float(inv_h2))
    assert abs(e0 - e_or) <= 1e-9 * abs(e_or)
    sim.run(400)
    e1 = sim.energy()
    assert e0 > 0 and abs(e1 - e0) / e0 < 1e-4
    sim.close()


# Receiver-IR error of 16-bit storage against the FP64 oracle on the
# 160x120x100 room over 600 steps, as measured (the GPU path equals the
# rounding oracle bit for bit, test_16bit_storage_bit_exact): FP16 5.6e-3,
# BF16 3.0e-2.  The regression bound is 1.25x the measured value; the
# accuracy target of 1e-3 is not met and is kept as a strict expected
# failure, so that a form that meets it shows up as an unexpected pass.
SMALL_16BIT_MEASURED = {capi.STORAGE_F16: 5.6e-3, capi.STORAGE_BF16: 3.0e-2}
IR_TARGET = 1e-3


def _small_16bit_error(storage):
    sc = scenes.plain_small(steps=600)
    g = oracle_grid(sc)
    want64 = oracle_scene(sc, g).run(sc.steps, f64=True)
    sim, _ = scenes.build_simulation(sc, storage=storage)
    sim.run(sc.steps)
    got = sim.ir()
    sim.close()
    assert np.isfinite(got).all()
    err = rel_l2(got, want64)
    print(f"storage {storage}: IR rel-L2 vs FP64 = {err:.3e}")
    return err


@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
def test_16bit_storage_error_regression(storage):
    assert _small_16bit_error(storage) <= 1.25 * SMALL_16BIT_MEASURED[storage]


@pytest.mark.xfail(strict=True, reason="16-bit storage: measured FP16 5.6e-3, BF16 3.0e-2 over 600 steps "
                                       "against the 1e-3 target (rounding of every stored value, every step)")
@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
def test_16bit_storage_error_meets_target(storage):
    assert _small_16bit_error(storage) <= IR_TARGET


def _storage_scale(sc) -> float:
    """The per-run scale the library chooses: the largest source amplitude
    maps to about 1024, rounded to a power of two."""
    peak = float(np.abs(sc.src_sig).max()) if sc.src_sig is not None and np.size(sc.src_sig) else 0.0
    if sc.hard is not None:
        peak = max(peak, float(np.abs(sc.hard).max()))
    return float(2.0 ** np.round(np.log2(1024.0 / peak))) if peak > 0 else 1.0


@pytest.mark.parametrize("storage", [capi.STORAGE_F16, capi.STORAGE_BF16])
@pytest.mark.parametrize("depth", [0, 2])
def test_16bit_storage_bit_exact(storage, depth):
    """16-bit storage against the oracle run that rounds every stored value
    the same way (FP32 update, the per-run scale): receiver samples and the
    final fields match bit for bit, for the register and the TMA kernels."""
    sc = scenes.plain_small(steps=400)
    g = oracle_grid(sc)
    scale = _storage_scale(sc)
    osc = oracle_scene(sc, g)
    osc.storage, osc.scale = storage, scale
    n = int(np.prod(g["shape"]))
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(g["bidx"].size * 12 + 1, np.float32))
    want = osc.run(sc.steps, state=st)
    sim, _ = scenes.build_simulation(sc, storage=storage, storage_scale=scale)
    sim.set_tiling(8, 0, depth)
    sim.run(sc.steps)
    got = sim.ir()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), np.abs(got - want).max()
    p = sim.pressure().reshape(-1)
    want_p = st[0] * np.float32(1.0 / scale)                    # unscaled on the GPU with flush-to-zero
    want_p[np.abs(want_p) < np.finfo(np.float32).tiny] *= np.float32(0.0)
    assert np.array_equal(p.view(np.uint32), want_p.view(np.uint32))
    sim.close()


def test_error_statuses():
    sim = capi.Simulation()
    with pytest.raises(capi.VirsError) as e:
        sim.classify()
    assert e.value.status == capi.E_STATE
    with pytest.raises(capi.VirsError) as e:
        sim.set_grid((8, 8, 8), 0.05, np.full(512, 4, np.uint8))
    assert e.value.status == capi.E_ARG
    sim.set_grid((8, 8, 8), 0.05, np.zeros(512, np.uint8))
    with pytest.raises(capi.VirsError) as e:
        sim.set_receivers([512])
    assert e.value.status == capi.E_ARG
    with pytest.raises(capi.VirsError) as e:
        sim.set_sources([0], np.ones((1, 4), np.float32))      # border voxel
    assert e.value.status == capi.E_ARG
    with pytest.raises(capi.VirsError) as e:
        sim.run(10)
    assert e.value.status == capi.E_STATE
    sim.classify()
    with pytest.raises(capi.VirsError) as e:
        sim.set_filters(np.full((1, 1, 5), np.nan, np.float32))
    assert e.value.status == capi.E_ARG
    with pytest.raises(capi.VirsError) as e:
        sim.set_tiling(5, 0)
    assert e.value.status == capi.E_ARG
    with pytest.raises(capi.VirsError) as e:
        capi.Simulation(capi.default_params(courant=1.5))
    assert e.value.status == capi.E_ARG
    with pytest.raises(capi.VirsError) as e:
        capi.Simulation(capi.default_params(sponge_width=40))
    assert e.value.status == capi.E_ARG
    with pytest.raises(capi.VirsError) as e:
        sim.load_obj("/nonexistent/room.obj")
    assert e.value.status == capi.E_IO
    sim.close()


def test_load_obj_matches_oracle_voxeliser(tmp_path):
    """An OBJ with an mtllib, quads and two materials (walls and a speaker),
    as Blender writes them; parsed by the library, voxelised and classified
    on the GPU; compared with the oracle on the same mesh."""
    sc = scenes.reference_room()
    (tmp_path / "room.mtl").write_text("newmtl Wall\nKd 0.8 0.8 0.8\n\nnewmtl Speaker\nKd 0.8 0 0\n")
    lines = ["mtllib room.mtl", "o Room"]
    for v in sc.verts:
        lines.append("v %.6f %.6f %.6f" % tuple(v))
    cur = None
    for t in range(0, len(sc.tris), 2):
        m = int(sc.tri_mat[t])
        if m != cur:
            lines.append("usemtl " + ("Wall" if m == 0 else "Speaker"))
            cur = m
        a, b, c = sc.tris[t] + 1
        d = sc.tris[t + 1][2] + 1
        lines.append(f"f {a}/1/1 {b}/1/1 {c}/1/1 {d}/1/1")
    (tmp_path / "room.obj").write_text("\n".join(lines) + "\n")
    p = capi.default_params(cell_size=sc.cell_size, bbox_nudge=sc.nudge)
    sim = capi.Simulation(p)
    sim.load_obj(tmp_path / "room.obj")
    sim.classify()
    verts = np.array([[float(x) for x in l.split()[1:]] for l in lines if l.startswith("v ")], np.float32)
    sc2 = dataclasses.replace(sc, verts=verts)
    g = oracle_grid(sc2)
    assert sim.shape == g["shape"]
    assert np.array_equal(sim.flags(), g["flags"])
    assert np.array_equal(sim.boundary_indices(), g["bidx"])
    assert np.count_nonzero(g["flags"] == 3) > 0
    sim.close()


def test_bounded_wait_reports_timeout_and_context_survives():
    """A wait that nothing completes gives up after its limit, the status is
    VIRS_E_TIMEOUT, and the same handle then runs normally."""
    sc = scenes.reference_room(steps=64)
    sim, _ = scenes.build_simulation(sc)
    assert sim.check_bounded_wait(2000) == capi.E_TIMEOUT
    sim.run(sc.steps)
    sim.synchronize()
    assert np.isfinite(sim.ir()).all()
    sim.close()


def test_autotune_keeps_results_bit_identical():
    sc = scenes.plain_small(steps=120)
    sim, _ = scenes.build_simulation(sc)
    sim.run(sc.steps)
    base = sim.ir()
    sim.start(sc.steps)
    t = sim.autotune(3)
    assert t.tile_rows in (4, 8, 16) and 1 <= t.pipeline_depth <= 3 and t.ms_per_step > 0
    assert sim.info().steps_done == 0
    sim.run(sc.steps)
    assert np.array_equal(sim.ir().view(np.uint32), base.view(np.uint32))
    got = sim.tiling()
    assert (got.tile_rows, got.planes_per_block, got.pipeline_depth) == (t.tile_rows, t.planes_per_block,
                                                                         t.pipeline_depth)
    sim.close()


@pytest.mark.parametrize("storage", [capi.STORAGE_F32, capi.STORAGE_BF16])
def test_batch_matches_members_run_alone(storage):
    """Three source positions in one room and three rooms of other sizes and
    materials, advanced together; every member's IR equals its own run."""
    scs = scenes.batched(steps=140, n_sources=3, n_rooms=3, room=64, size_range=(40, 90))
    alone = []
    for sc in scs:
        sim, _ = scenes.build_simulation(sc, storage=storage)
        sim.run(sc.steps)
        alone.append(sim.ir())
        sim.close()
    sims = [scenes.build_simulation(sc, storage=storage)[0] for sc in scs]
    with capi.Batch(sims) as b:
        b.run(100)              # graph chunks + remainder
        b.run(40)
        b.synchronize()
        for sim, want in zip(sims, alone):
            assert np.array_equal(sim.ir().view(np.uint32), want.view(np.uint32))
    for s in sims:
        s.close()


def test_batch_rejects_changed_members():
    scs = scenes.batched(steps=20, n_sources=2, n_rooms=0, room=48)
    sims = [scenes.build_simulation(sc)[0] for sc in scs]
    b = capi.Batch(sims)
    sims[1].set_receivers([int(sims[1].boundary_indices()[0])])
    with pytest.raises(capi.VirsError) as e:
        b.run(4)
    assert e.value.status == capi.E_STATE
    b.close()
    for s in sims:
        s.close()


def test_gpu_voxeliser_overlapping_triangles_match_oracle():
    """A shoebox plus 80 seeded triangles of five materials (three wall
    absorbers, a speaker, an ignored one) that overlap each other: the last
    triangle in mesh order decides a voxel's flag, the last wall triangle its
    material, whatever order the GPU visits them in."""
    rng = np.random.default_rng(11)
    base = scenes.reference_room()
    L = base.verts.max(0) - base.verts.min(0)
    lo = base.verts.min(0)
    verts = [base.verts]
    tris = [base.tris]
    mats = [base.tri_mat]
    n0 = len(base.verts)
    for t in range(80):
        c = lo + L * rng.uniform(0.15, 0.85, 3)
        v = (c + rng.normal(0, 0.12, (3, 3)) * L.min()).astype(np.float32)
        verts.append(v)
        tris.append(np.arange(3, dtype=np.uint32)[None, :] + n0)
        mats.append(np.array([rng.integers(0, 5)], np.int32))
        n0 += 3
    roles = np.array([0, capi.ROLE_SOURCE, 1, capi.ROLE_IGNORE, 2], np.uint8)
    sc = dataclasses.replace(base, verts=np.concatenate(verts).astype(np.float32),
                             tris=np.concatenate(tris).astype(np.uint32), tri_mat=np.concatenate(mats).astype(np.int32),
                             roles=roles, sponge_width=2, n_materials=3)
    g = oracle_grid(sc)
    sim = capi.Simulation(capi.default_params(cell_size=sc.cell_size, bbox_nudge=sc.nudge, sponge_width=2))
    sim.set_material_roles(sc.roles)
    sim.set_mesh(sc.verts, sc.tris, sc.tri_mat)
    sim.classify()
    assert np.count_nonzero(g["flags"] == 3) > 0 and np.count_nonzero(g["flags_raw"] == 1) > 0
    _grid_parity(sim, g)
    sim.close()


@pytest.mark.parametrize("storage", [capi.STORAGE_F32, capi.STORAGE_BF16])
@pytest.mark.parametrize("rows,planes", [(8, 16), (16, 64)])
def test_wide_grid_skips_zero_code_planes_bit_exact(storage, rows, planes):
    """A hall three tiles wide (384 voxels): the middle tile column has
    planes whose codes are all zero, which the TMA stencil does not copy.
    Receiver samples and fields still equal the oracle's bit for bit."""
    sc = scenes.large_hall(steps=300, size=(384, 80, 72))
    g = oracle_grid(sc)
    osc = oracle_scene(sc, g)
    scale = 1.0
    if storage != capi.STORAGE_F32:
        scale = _storage_scale(sc)
        osc.storage, osc.scale = storage, scale
    n = int(np.prod(g["shape"]))
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(g["bidx"].size * 12 + 1, np.float32))
    want = osc.run(sc.steps, state=st)
    sim, _ = scenes.build_simulation(sc, storage=storage, storage_scale=scale if storage else 0.0)
    sim.set_tiling(rows, planes, 2)
    sim.run(sc.steps)
    got = sim.ir()
    assert np.abs(want).max() > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), np.abs(got - want).max()
    p = sim.pressure().reshape(-1)
    want_p = st[0] * np.float32(1.0 / scale)
    if storage != capi.STORAGE_F32:
        want_p[np.abs(want_p) < np.finfo(np.float32).tiny] *= np.float32(0.0)
    assert np.array_equal(p.view(np.uint32), want_p.view(np.uint32))
    sim.close()


@pytest.mark.parametrize("storage", [capi.STORAGE_F32, capi.STORAGE_BF16])
def test_init_sphere_matches_oracle(storage):
    """virs_init_pressure_sphere against the oracle's restatement of
    initSphereKernel (init_sphere.cu:4-25): spheres inside the grid, cut by
    its faces and of radius 0, with and without zeroing the rest.  The
    library keeps the domain border at 0 (the step never writes it, so a
    pressure there would stay for ever); every interior voxel must equal the
    oracle's, and p^{n-1} is left alone, as in the reference."""
    shape = (37, 29, 23)
    nx, ny, nz = shape
    n = nx * ny * nz
    rng = np.random.default_rng(11)
    sim = capi.Simulation(storage=storage, storage_scale=1.0 if storage else 0.0)
    sim.set_grid(shape, 0.05, np.zeros(n, np.uint8))
    sim.classify()
    sim.start(1)
    interior = np.zeros((nz, ny, nx), bool)
    interior[1:-1, 1:-1, 1:-1] = True
    interior = interior.reshape(-1)
    cases = [((18, 14, 11), 5, 1.25, True), ((1, 2, 3), 7, -0.5, False), ((36, 28, 22), 11, 2.0, False),
             ((10, 10, 10), 0, 3.0, False), ((0, 14, 11), 3, 0.75, True)]
    for center, radius, value, zero in cases:
        base = rng.integers(-8, 8, n).astype(np.float32) / 4      # exact in BF16
        base[~interior] = 0
        prev = rng.integers(-8, 8, n).astype(np.float32) / 4
        prev[~interior] = 0
        sim.set_pressure(base, prev)
        sim.init_pressure_sphere(*center, radius, value, zero)
        got, got_prev = sim.pressure(prev=True)
        want = oracle.init_sphere(base.copy(), shape, center, radius, value, zero)
        assert np.array_equal(got[interior], want[interior]), (center, radius)
        assert not got[~interior].any()
        assert np.array_equal(got_prev, prev)
    sim.close()
