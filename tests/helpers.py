"""Shared test helpers: build the same scene for the oracle and for the GPU."""
from __future__ import annotations

import numpy as np

import oracle
from virs_b200 import scenes


def oracle_grid(sc: scenes.Scene):
    """Voxelise + classify a scene with the oracle.  Returns a dict."""
    tris = sc.verts[sc.tris].reshape(-1, 9)
    lo, hi = oracle.bbox(sc.verts, sc.nudge)
    h = float(np.float32(sc.cell_size))
    shape = oracle.dims(lo, hi, h)
    flags0, wmat = oracle.voxelize(tris, sc.tri_mat, sc.roles, h, lo, shape)
    flags, bmat_full, bd2_full = oracle.classify(shape, sc.sponge_width, flags0, wmat)
    bidx = oracle.boundary_list(shape, flags)
    bmat = bmat_full[bidx]
    bw = oracle.sponge_weights_for(sc.sponge_width, bd2_full[bidx])
    return dict(shape=shape, bmin=lo, h=h, flags_raw=flags0, wall_mat=wmat, flags=flags, bidx=bidx,
                bmat=bmat, bw=bw, normals=oracle.normals(shape, flags))


def oracle_scene(sc: scenes.Scene, g: dict, *, K=None, f64_coef=None):
    """oracle.Scene for a run of `sc` on grid `g`."""
    dt, c2dt2, inv_h2, Kf = oracle.step_constants(g["h"], 343.0, sc.courant)
    if K is not None:
        Kf = np.float32(K)
    if sc.coef64 is None:
        fs = oracle.filter_fs(g["h"], 343.0, sc.courant)
        c32 = oracle.rbj_highpass_ref(fs, 440.0, 0.1)[None, None, :]
        c64 = c32.astype(np.float64)
    else:
        c32 = sc.coef64.astype(np.float32)
        c64 = sc.coef64
    src_idx = scenes.voxel_index(sc.src_pos, g["bmin"], g["h"], g["shape"]) if len(sc.src_pos) else np.zeros(0, np.uint64)
    rcv_idx = scenes.voxel_index(sc.rcv_pos, g["bmin"], g["h"], g["shape"]) if len(sc.rcv_pos) else np.zeros(0, np.uint64)
    hard = np.full(10, 10.0, np.float32) if sc.hard is None else sc.hard
    c2d, ih2d = float(c2dt2), float(inv_h2)
    return oracle.Scene(g["shape"], g["flags"], g["bidx"], g["bmat"], g["bw"], c32, c32.shape[1] if c32.ndim == 3 else 1,
                        coef64=c64, hard=hard, src_idx=src_idx, src_sig=sc.src_sig, rcv_idx=rcv_idx,
                        consts=(c2dt2, inv_h2, Kf), consts64=(c2d, ih2d, float(Kf)), form=scenes.boundary_form(sc))


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def grid_parity(sim, g: dict) -> None:
    """A classified simulation's grid against the oracle's: shape, flags,
    normals, boundary list, and each boundary voxel's material and sponge
    weight, all bit for bit."""
    assert sim.shape == tuple(g["shape"])
    assert np.array_equal(sim.flags(), g["flags"])
    assert np.array_equal(sim.normals(), g["normals"])
    assert np.array_equal(sim.boundary_indices(), g["bidx"])
    m, w = sim.boundary_materials()
    assert np.array_equal(m, g["bmat"])
    assert np.array_equal(w.view(np.uint32), g["bw"].view(np.uint32))
