"""z-slabs on one GPU: a grid split into slab handles whose ghost planes are
refreshed from their neighbours before every step advances exactly as the
whole grid, bit for bit: classification of the owned planes (flags,
normals, boundary list, materials, weights), receiver samples and fields.

The exchange here is `slabs.exchange_local` (device copies on the current
stream between handles of one process); across processes the same planes
go through torch.distributed (`slabs.exchange`, covered on CPU by
test_slabs.py)."""
import dataclasses

import numpy as np
import pytest

import oracle
from virs_b200 import capi, scenes, slabs

pytestmark = pytest.mark.gpu


def _scene(steps):
    # boxes, 4 materials, 3-section cascades; sponge 6 so the classification
    # halo of the slabs matters; a soft source and receivers spread in z
    sc = scenes.furnished_room(steps=steps)
    return dataclasses.replace(sc, cell_size=1 / 32, sponge_width=6)


def test_mesh_slab_flags_equal_whole_grid():
    """Each slab voxelises only its planes of the mesh (global origin and
    sizes): its flags and wall materials equal the whole grid's planes."""
    sc = _scene(10)
    p = capi.default_params(courant=sc.courant, cell_size=sc.cell_size, bbox_nudge=sc.nudge,
                            sponge_width=sc.sponge_width)
    with capi.Simulation(p) as whole:
        whole.set_material_roles(sc.roles)
        whole.set_mesh(sc.verts, sc.tris, sc.tri_mat)
        wf, wm = whole.flags(), whole.wall_materials()
        nx, ny, nz = whole.shape
        bmin = list(whole.info().bbox_min)
    # the whole grid's voxelisation is the oracle's
    lo, _ = oracle.bbox(sc.verts, sc.nudge)
    of, ow = oracle.voxelize(sc.verts[sc.tris].reshape(-1, 9), sc.tri_mat, sc.roles, float(np.float32(sc.cell_size)),
                             lo, (nx, ny, nz))
    assert np.array_equal(wf, of) and np.array_equal(wm, ow)
    plane = nx * ny
    for part in range(3):
        with capi.Simulation(p) as s:
            s.set_material_roles(sc.roles)
            s.set_mesh_slab(sc.verts, sc.tris, sc.tri_mat, part, 3)
            z_lo, z_hi, n = s.slab_info()
            assert (n, (z_lo, z_hi)) == (nz, slabs.split_planes(nz, 3)[part])
            assert s.shape == (nx, ny, z_hi - z_lo + 2)
            assert list(s.info().bbox_min) == bmin
            keep = slice((z_lo - 1) * plane, (z_hi + 1) * plane)
            assert np.array_equal(s.flags(), wf[keep])
            assert np.array_equal(s.wall_materials(), wm[keep])


def _run_slabs(parts, steps):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(steps):
        slabs.exchange_local([p[0] for p in parts])
        for s, *_ in parts:
            s.run(1, stream=stream)
    torch.cuda.synchronize()


@pytest.mark.parametrize("nparts,voxelise", [(2, "whole"), (3, "slab")])
def test_slabs_match_whole_grid_f32(nparts, voxelise):
    sc = _scene(240)
    whole, meta = scenes.build_simulation(sc)
    nx, ny, nz = meta["shape"]
    plane = nx * ny
    wf, wn, wb = whole.flags(), whole.normals(), whole.boundary_indices()
    wm, ww = whole.boundary_materials()
    parts, pmeta = scenes.build_slabs(sc, nparts, voxelise=voxelise)
    assert pmeta["shape"] == meta["shape"]
    got_b, got_m, got_w = [], [], []
    for s, z_lo, z_hi, _ in parts:
        assert s.shape == (nx, ny, z_hi - z_lo + 2)
        own = slice(plane, (z_hi - z_lo + 1) * plane)       # local planes 1 .. nz_local-2
        gown = slice(z_lo * plane, z_hi * plane)
        assert np.array_equal(s.flags()[own], wf[gown])
        assert np.array_equal(s.normals()[own], wn[gown])
        b = s.boundary_indices().astype(np.int64) + (z_lo - 1) * plane
        m, w = s.boundary_materials()
        got_b.append(b)
        got_m.append(m)
        got_w.append(w)
    # the slabs' boundary lists, in slab order, are the whole grid's list
    assert np.array_equal(np.concatenate(got_b), wb.astype(np.int64))
    assert np.array_equal(np.concatenate(got_m), wm)
    assert np.array_equal(np.concatenate(got_w).view(np.uint32), ww.view(np.uint32))

    whole.run(sc.steps)
    want_ir = whole.ir()
    want_p, want_pp = whole.pressure(prev=True)
    _run_slabs(parts, sc.steps)
    ir = np.zeros_like(want_ir)
    for s, z_lo, z_hi, own_r in parts:
        if own_r.any():
            ir[own_r] = s.ir()
        p, pp = s.pressure(prev=True)
        gown = slice(z_lo * plane, z_hi * plane)
        assert np.array_equal(p[plane:(z_hi - z_lo + 1) * plane].view(np.uint32), want_p[gown].view(np.uint32))
        assert np.array_equal(pp[plane:(z_hi - z_lo + 1) * plane].view(np.uint32), want_pp[gown].view(np.uint32))
    assert sum(int(o.sum()) for *_, o in parts) == want_ir.shape[0]
    assert np.abs(want_ir).max() > 0
    assert np.array_equal(ir.view(np.uint32), want_ir.view(np.uint32))
    for s, *_ in parts:
        s.close()
    whole.close()


def test_slabs_match_whole_grid_bf16():
    """16-bit storage with the same explicit scale on every handle."""
    sc = _scene(160)
    scale = 64.0
    whole, meta = scenes.build_simulation(sc, storage=capi.STORAGE_BF16, storage_scale=scale)
    parts, _ = scenes.build_slabs(sc, 2, storage=capi.STORAGE_BF16, storage_scale=scale)
    whole.run(sc.steps)
    want_ir = whole.ir()
    _run_slabs(parts, sc.steps)
    ir = np.zeros_like(want_ir)
    for s, _, _, own_r in parts:
        if own_r.any():
            ir[own_r] = s.ir()
    assert np.abs(want_ir).max() > 0
    assert np.array_equal(ir.view(np.uint32), want_ir.view(np.uint32))
    for s, *_ in parts:
        s.close()
    whole.close()


def test_slab_arguments_checked():
    sc = _scene(10)
    with capi.Simulation(capi.default_params(sponge_width=6)) as s:
        flags = np.zeros((40, 8, 8), np.uint8)
        # owned planes outside 1 .. nz-2
        with pytest.raises(capi.VirsError):
            s.set_grid_slab((8, 8, 40), 0.1, 0, 10, flags)
        # flags that miss the classification halo (W + 1 = 7 planes beyond the ghost)
        with pytest.raises(capi.VirsError):
            s.set_grid_slab((8, 8, 40), 0.1, 20, 30, flags[12:32], z_first=12)
        s.set_grid_slab((8, 8, 40), 0.1, 20, 30, flags[12:38], z_first=12)
        assert s.shape == (8, 8, 12)
        first, last, glo, ghi, nb = s.slab_planes()
        assert nb == 32 * 8 * 4 and first - glo == nb and ghi - last == nb
    with capi.Simulation(capi.default_params(storage=capi.STORAGE_BF16)) as s:
        with pytest.raises(capi.VirsError):  # 16-bit slabs need an explicit scale
            s.set_grid_slab((8, 8, 40), 0.1, 1, 20, np.zeros((40, 8, 8), np.uint8))
    del sc


def _build_slab_room(tmp_path):
    import shutil
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = tmp_path / "slab_room"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{root / 'include'}",
           str(root / "tests" / "cpp" / "slab_room.cpp"), f"-L{root / 'virs_b200'}", "-lvirs_b200",
           f"-Wl,-rpath,{root / 'virs_b200'}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.parametrize("parts,storage", [(2, 0), (3, 0), (3, 2)])
def test_slab_run_from_cpp_matches_whole_grid(tmp_path, parts, storage):
    """A C++ host drives the slabs through the C ABI (virs_set_mesh_slab,
    virs_slab_run: the library exchanges the ghost planes before every
    step): receiver samples and owned planes equal the whole grid's."""
    import subprocess
    exe = _build_slab_room(tmp_path)
    r = subprocess.run([str(exe), str(parts), "200", str(storage)], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    assert r.returncode == 0, r.stderr
    assert "equal" in r.stdout


def test_slab_exchange_arguments_checked():
    sc = _scene(10)
    parts, _ = scenes.build_slabs(sc, 3)
    a, b, c = (p[0] for p in parts)
    with pytest.raises(capi.VirsError) as e:
        capi.slab_exchange(a, c)                       # not adjacent
    assert e.value.status == capi.E_ARG
    with pytest.raises(capi.VirsError) as e:
        capi.slab_run([a, b], 1)                       # does not cover the grid
    assert e.value.status == capi.E_ARG
    capi.slab_run([a, b, c], 2)
    b.run(1)                                           # one slab a step ahead
    with pytest.raises(capi.VirsError) as e:
        capi.slab_exchange(b, c)
    assert e.value.status == capi.E_STATE
    for s in (a, b, c):
        s.close()


@pytest.mark.parametrize("parts", [3, 7])
def test_slab_run_thin_slabs_match_whole_grid(parts):
    """virs_slab_run on slabs that own one to three planes: the interior
    launch (planes 2 .. nz-3) is empty or a single plane, and the edge planes
    are one plane or two.  A 64x48x9 hall: 7 interior planes.  The run of
    49 steps replays the 16-step graph of the odd buffer parity three times,
    the run of 30 the graph of the even parity once, each followed by direct
    launches."""
    sc = scenes.large_hall(steps=80, size=(64, 48, 9))
    whole, meta = scenes.build_simulation(sc)
    whole.run(sc.steps)
    want_ir = whole.ir()
    want_p, want_pp = whole.pressure(prev=True)
    nx, ny, _ = meta["shape"]
    plane = nx * ny
    parts_, _ = scenes.build_slabs(sc, parts)
    sims = [p[0] for p in parts_]
    capi.slab_run(sims, 1)
    capi.slab_run(sims, 49)
    capi.slab_run(sims, 30)
    ir = np.zeros_like(want_ir)
    for s, z_lo, z_hi, own_r in parts_:
        s.synchronize()
        if own_r.any():
            ir[own_r] = s.ir()
        p, pp = s.pressure(prev=True)
        gown = slice(z_lo * plane, z_hi * plane)
        assert np.array_equal(p[plane:(z_hi - z_lo + 1) * plane].view(np.uint32), want_p[gown].view(np.uint32))
        assert np.array_equal(pp[plane:(z_hi - z_lo + 1) * plane].view(np.uint32), want_pp[gown].view(np.uint32))
    assert np.abs(want_ir).max() > 0
    assert np.array_equal(ir.view(np.uint32), want_ir.view(np.uint32))
    for s in sims:
        s.close()
    whole.close()


@pytest.mark.parametrize("nparts,storage,rounding", [(2, capi.STORAGE_F32, capi.ROUND_NEAREST),
                                                    (3, capi.STORAGE_BF16, capi.ROUND_NEAREST),
                                                    (2, capi.STORAGE_F16, capi.ROUND_STOCHASTIC)])
def test_split_slab_step_matches_whole_grid(nparts, storage, rounding):
    """virs_slab_step_begin / virs_slab_step_end with the ghost planes
    exchanged between the two parts (the form a multi-process host uses,
    here with device copies in one process): the interior launches of
    every slab run on a side stream while the copies run on the main one;
    receivers and owned planes equal the whole grid's bit for bit (with
    stochastic rounding too: a slab's voxels take the whole grid's keys)."""
    import torch
    sc = _scene(150)
    scale = 64.0 if storage else 0.0
    whole, meta = scenes.build_simulation(sc, storage=storage, storage_scale=scale)
    whole.set_rounding(rounding)
    nx, ny, _ = meta["shape"]
    plane = nx * ny
    whole.run(sc.steps)
    want_ir = whole.ir()
    want_p, want_pp = whole.pressure(prev=True)
    parts, _ = scenes.build_slabs(sc, nparts, storage=storage, storage_scale=scale)
    sims = [p[0] for p in parts]
    for s in sims:
        s.set_rounding(rounding)
    main = torch.cuda.current_stream()
    side = torch.cuda.Stream()
    for _ in range(sc.steps):
        side.wait_stream(main)
        for s in sims:
            s.slab_step_begin(side.cuda_stream)
        slabs.exchange_local(sims)
        main.wait_stream(side)
        for s in sims:
            s.slab_step_end(main.cuda_stream)
    torch.cuda.synchronize()
    ir = np.zeros_like(want_ir)
    for s, z_lo, z_hi, own_r in parts:
        if own_r.any():
            ir[own_r] = s.ir()
        p, pp = s.pressure(prev=True)
        gown = slice(z_lo * plane, z_hi * plane)
        assert np.array_equal(p[plane:(z_hi - z_lo + 1) * plane].view(np.uint32), want_p[gown].view(np.uint32))
        assert np.array_equal(pp[plane:(z_hi - z_lo + 1) * plane].view(np.uint32), want_pp[gown].view(np.uint32))
    assert np.abs(want_ir).max() > 0
    assert np.array_equal(ir.view(np.uint32), want_ir.view(np.uint32))
    for s in sims:
        s.close()
    whole.close()


def test_split_slab_step_order_checked():
    """A second begin, a run, or an end without a begin is refused, and the
    handle stays usable."""
    import torch
    st = torch.cuda.current_stream().cuda_stream
    sc = _scene(20)
    parts, _ = scenes.build_slabs(sc, 2)
    a, b = (p[0] for p in parts)
    with pytest.raises(capi.VirsError) as e:
        a.slab_step_end(st)
    assert e.value.status == capi.E_STATE
    a.slab_step_begin(st)
    with pytest.raises(capi.VirsError) as e:
        a.slab_step_begin(st)
    assert e.value.status == capi.E_STATE
    with pytest.raises(capi.VirsError) as e:
        a.run(1)
    assert e.value.status == capi.E_STATE
    with pytest.raises(capi.VirsError) as e:
        capi.slab_run([a, b], 1)
    assert e.value.status == capi.E_STATE
    b.slab_step_begin(st)
    slabs.exchange_local([a, b])
    a.slab_step_end(st)
    b.slab_step_end(st)
    capi.slab_run([a, b], 3)
    for s in (a, b):
        s.synchronize()
        assert s.info().steps_done == 4
        s.close()


def test_slab_run_class_single_rank_matches_whole_grid():
    """slabs.SlabRun on one rank (the grid as one slab, no neighbours, so no
    collective): the interior launch on its side stream and the end of the
    step on the current stream give the whole grid's results bit for bit."""
    sc = _scene(80)
    whole, _ = scenes.build_simulation(sc)
    whole.run(sc.steps)
    want_ir = whole.ir()
    parts, _ = scenes.build_slabs(sc, 1)
    sim = parts[0][0]
    slabs.SlabRun(sim, 0, 1).run(sc.steps)
    sim.synchronize()
    got = sim.ir()
    assert np.abs(want_ir).max() > 0
    assert np.array_equal(got.view(np.uint32), want_ir.view(np.uint32))
    sim.close()
    whole.close()
