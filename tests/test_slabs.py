"""z-slab host logic on CPU: the split of the planes, the flag ranges for the
classification halo, voxel index mapping, and the halo exchange between
two gloo ranks.  Each rank steps the oracle on its slab (classified from
its extended planes, then cut to its planes and two ghost planes) and
refreshes the ghost planes from the other rank with `slabs.exchange` before
every step; together they must equal the oracle on the whole grid bit for
bit."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from virs_b200 import slabs

ROOT = Path(__file__).resolve().parents[1]
W = 3          # sponge width: the classification halo is W + 1 planes
STEPS = 120


def test_split_planes():
    assert slabs.split_planes(10, 1) == [(1, 9)]
    assert slabs.split_planes(10, 3) == [(1, 4), (4, 7), (7, 9)]
    parts = slabs.split_planes(515, 8)
    assert parts[0][0] == 1 and parts[-1][1] == 514
    assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
    assert max(b - a for a, b in parts) - min(b - a for a, b in parts) <= 1
    with pytest.raises(ValueError):
        slabs.split_planes(4, 3)


def test_flag_range_and_local_index():
    assert slabs.flag_range(100, 1, 34, 6) == (0, 42)       # bottom slab: from the border plane
    assert slabs.flag_range(100, 34, 67, 6) == (26, 49)
    assert slabs.flag_range(100, 67, 99, 6) == (59, 41)     # top slab: to the border plane
    shape = (5, 4, 10)
    idx = np.array([0, 5 * 4 * 3 + 7, 5 * 4 * 6, 5 * 4 * 9 - 1], np.uint64)   # planes 0, 3, 6, 8
    own, loc = slabs.local_index(idx, shape, 3, 6)
    assert own.tolist() == [False, True, False, False]
    assert loc.tolist() == [5 * 4 * 1 + 7]                     # local plane 1 = global plane 3


def _grid():
    """A shoebox with an interior box that crosses the split, two wall
    materials, a hard-source voxel in the upper half."""
    nx, ny, nz = 20, 18, 26
    f = np.zeros((nz, ny, nx), np.uint8)
    wm = np.zeros_like(f)
    f[1, 1:-1, 1:-1] = 1
    f[nz - 2, 1:-1, 1:-1] = 1
    f[1:-1, 1, 1:-1] = 1
    f[1:-1, ny - 2, 1:-1] = 1
    f[1:-1, 1:-1, 1] = 1
    f[1:-1, 1:-1, nx - 2] = 1
    f[10:16, 6:10, 7:11] = 1
    wm[f == 1] = 0
    wm[nz - 2][f[nz - 2] == 1] = 1
    wm[10:16, 6:10, 7:11] = 1
    f[18, 12, 13] = 3
    return (nx, ny, nz), f.reshape(-1), wm.reshape(-1)


def _classified(shape, flags, wmat):
    fo, bm, bd = oracle.classify(shape, W, flags, wmat)
    return fo, bm, bd


def _scene(shape, fo, bm, bd, src_idx, rcv_idx, sig):
    h = 0.05
    _, c2dt2, inv_h2, K = oracle.step_constants(h, 343.0, 0.5)
    fs = oracle.filter_fs(h, 343.0, 0.5)
    coef = np.stack([oracle.rbj_highpass_ref(fs, 440.0, 0.1), oracle.rbj_highpass_ref(fs, 1200.0, 0.3)])[:, None, :]
    bidx = oracle.boundary_list(shape, fo)
    return oracle.Scene(shape, fo, bidx, bm[bidx], oracle.sponge_weights_for(W, bd[bidx]), coef, 1,
                        hard=np.full(10, 10.0, np.float32), src_idx=src_idx, src_sig=sig, rcv_idx=rcv_idx,
                        consts=(c2dt2, inv_h2, K))


def _sources(shape):
    nx, ny, _ = shape
    src = np.array([(7 * ny + 9) * nx + 12], np.uint64)                         # plane 7
    rcv = np.array([(4 * ny + 5) * nx + 5, (12 * ny + 4) * nx + 14, (20 * ny + 9) * nx + 9], np.uint64)
    t = np.arange(STEPS, dtype=np.float64)
    sig = (-(t - 24) / 8.0 * np.exp(-0.5 * ((t - 24) / 8.0) ** 2)).astype(np.float32)[None, :]
    return src, rcv, sig


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        shape, flags, wmat = _grid()
        nx, ny, nz = shape
        plane = nx * ny
        z_lo, z_hi = slabs.split_planes(nz, world)[rank]
        z_first, n_ext = slabs.flag_range(nz, z_lo, z_hi, W)
        ext = slice(z_first * plane, (z_first + n_ext) * plane)
        fo, bm, bd = _classified((nx, ny, n_ext), flags[ext], wmat[ext])
        keep = slice((z_lo - 1 - z_first) * plane, (z_hi + 1 - z_first) * plane)
        lshape = (nx, ny, z_hi - z_lo + 2)
        src, rcv, sig = _sources(shape)
        own_s, loc_s = slabs.local_index(src, shape, z_lo, z_hi)
        own_r, loc_r = slabs.local_index(rcv, shape, z_lo, z_hi)
        osc = _scene(lshape, fo[keep], bm[keep], bd[keep], loc_s, loc_r, sig[own_s])
        n = int(np.prod(lshape))
        p, pp = np.zeros(n, np.float32), np.zeros(n, np.float32)
        st = np.zeros(max(osc.bidx.size * 4, 1), np.float32)
        P = p.reshape(-1, plane)
        ir = []
        for k in range(STEPS):
            slabs.exchange(torch.from_numpy(P[1]), torch.from_numpy(P[-2]), torch.from_numpy(P[0]),
                           torch.from_numpy(P[-1]), rank, world)
            ir.append(osc.run(1, state=(p, pp, st), step0=k))
        ir = np.concatenate(ir, axis=1) if loc_r.size else np.zeros((0, STEPS), np.float32)
        out[rank] = (z_lo, z_hi, p[plane:-plane].copy(), own_r, ir)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_whole_grid():
    shape, flags, wmat = _grid()
    nx, ny, nz = shape
    plane = nx * ny
    fo, bm, bd = _classified(shape, flags, wmat)
    src, rcv, sig = _sources(shape)
    whole = _scene(shape, fo, bm, bd, src, rcv, sig)
    p = np.zeros(int(np.prod(shape)), np.float32)
    state = (p, np.zeros_like(p), np.zeros(max(whole.bidx.size * 4, 1), np.float32))
    want_ir = whole.run(STEPS, state=state)
    assert np.abs(want_ir).max() > 1e-3

    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    ir = np.zeros_like(want_ir)
    for r in range(world):
        z_lo, z_hi, owned, own_r, rir = res[r]
        assert np.array_equal(owned.view(np.uint32), p[z_lo * plane:z_hi * plane].view(np.uint32))
        ir[own_r] = rir
    assert np.array_equal(ir.view(np.uint32), want_ir.view(np.uint32))
