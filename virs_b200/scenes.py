"""Seeded synthetic scenes for the FDTD path.

There are no public datasets for this path; every workload is generated here
from a documented seed: axis-aligned room meshes (12 triangles per box, the
shape of a Blender-exported shoebox), per-face OBJ material ids, source
signals, receiver positions, and absorbing-filter designs.

Workloads (sizes as the benchmark configurations name them):
  plain_small      4.0 x 3.0 x 2.5 m shoebox at h = 0.025 m -> 160x120x100,
                   Courant 1/sqrt(3), 6 walls with one first-order absorber
                   each (reflection uniform in [0.6, 0.95]), sponge width 8,
                   differentiated-Gaussian source (sigma 8 steps), 1 receiver,
                   2000 steps
  furnished_room   8 x 6 x 3 m shoebox + 20 boxes (0.3-2 m) at h = 1/64 m ->
                   512x384x192, 4 materials of 3-section octave cascades
                   (absorption in [0.05, 0.8]), sponge 16, 4 receivers, 10000
                   steps
  large_hall       16 x 12 x 8 m hall at h = 1/64 m -> 1024x768x512, 2
                   materials of 3-section cascades, Gaussian pulse source, 8
                   receivers, 4000 steps, sponge width 1
  reference_room   the reference's defaults on a small grid: one material, RBJ
                   high-pass 440 Hz Q 0.1, a speaker box voxelised as hard
                   source (flag 3, 10 for 10 steps), sponge 1, Courant 0.5/sqrt 3
"""
from __future__ import annotations

import contextlib
from dataclasses import dataclass, field

import numpy as np

# face order of box(): -x, +x, -y, +y, -z, +z (two triangles each)
FACES = ("-x", "+x", "-y", "+y", "-z", "+z")


def box(lo, hi, face_materials):
    """Axis-aligned box as 8 vertices and 12 triangles; face_materials is one
    OBJ material id per face (FACES order) or one id for all faces."""
    x0, y0, z0 = (float(v) for v in lo)
    x1, y1, z1 = (float(v) for v in hi)
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x0, y1, z0], [x1, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x0, y1, z1], [x1, y1, z1]], np.float32)
    quads = [(0, 2, 6, 4), (1, 5, 7, 3), (0, 4, 5, 1), (2, 3, 7, 6), (0, 1, 3, 2), (4, 6, 7, 5)]
    fm = np.broadcast_to(np.asarray(face_materials, np.int32), (6,))
    tris, mats = [], []
    for q, m in zip(quads, fm):
        tris += [(q[0], q[1], q[2]), (q[0], q[2], q[3])]
        mats += [m, m]
    return v, np.array(tris, np.uint32), np.array(mats, np.int32)


def merge(*meshes):
    vs, ts, ms, off = [], [], [], 0
    for v, t, m in meshes:
        vs.append(v)
        ts.append(t + off)
        ms.append(m)
        off += v.shape[0]
    return np.concatenate(vs), np.concatenate(ts), np.concatenate(ms)


def diff_gaussian(n: int, sigma: float, amp: float = 1.0, delay: float | None = None) -> np.ndarray:
    """Differentiated Gaussian pulse -(t - t0)/sigma^2 exp(-(t - t0)^2 / 2 sigma^2),
    scaled to peak |amp|, t in steps, t0 = 4 sigma."""
    t0 = 4.0 * sigma if delay is None else delay
    t = np.arange(n, dtype=np.float64)
    s = -(t - t0) / sigma**2 * np.exp(-((t - t0) ** 2) / (2 * sigma**2))
    return (amp * s / np.abs(s).max()).astype(np.float32)


def gaussian(n: int, sigma: float, amp: float = 1.0, delay: float | None = None) -> np.ndarray:
    t0 = 4.0 * sigma if delay is None else delay
    t = np.arange(n, dtype=np.float64)
    return (amp * np.exp(-((t - t0) ** 2) / (2 * sigma**2))).astype(np.float32)


@dataclass
class Scene:
    """A complete workload: mesh, parameters, filters, sources, receivers."""
    name: str
    verts: np.ndarray
    tris: np.ndarray
    tri_mat: np.ndarray
    roles: np.ndarray
    cell_size: float
    nudge: float
    courant: float
    sponge_width: int
    steps: int
    n_materials: int
    n_sections: int
    coef64: np.ndarray | None = None       # [M][S][5] FP64 design (None = reference high-pass)
    src_pos: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))   # world metres
    src_sig: np.ndarray | None = None      # [n_src][steps]
    rcv_pos: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    hard: np.ndarray | None = None         # flag-3 schedule (None = reference 10 x 10)
    seed: int = 0

    @property
    def coef32(self):
        return None if self.coef64 is None else self.coef64.astype(np.float32)


def _interior_points(rng, lo, hi, n, margin):
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    m = np.minimum(margin, 0.25 * (hi - lo))       # thin crops keep a quarter on each side
    return rng.uniform(lo + m, hi - m, (n, 3))


def plain_small(seed: int = 1, steps: int = 2000) -> Scene:
    rng = np.random.default_rng(seed)
    L = (4.0, 3.0, 2.5)
    h = 0.025
    v, t, m = box((0, 0, 0), L, np.arange(6))
    fs = fs_of(h, 1.0)
    R = rng.uniform(0.6, 0.95, 6)
    coef = np.stack([design_first_order_np(fs, r, 1000.0) for r in R])[:, None, :]
    src = _interior_points(rng, (0, 0, 0), L, 1, 0.5)
    rcv = _interior_points(rng, (0, 0, 0), L, 1, 0.5)
    sig = diff_gaussian(steps, 8.0)[None, :]
    return Scene("plain_small", v, t, m, np.arange(6, dtype=np.uint8), h, 0.0, 1.0, 8, steps, 6, 1, coef,
                 src, sig, rcv, seed=seed)


def furnished_room(seed: int = 2, steps: int = 10000, n_boxes: int = 20) -> Scene:
    rng = np.random.default_rng(seed)
    L = np.array([8.0, 6.0, 3.0])
    h = 1.0 / 64.0
    meshes = [box((0, 0, 0), L, [2, 2, 3, 3, 0, 1])]      # walls 2/3, floor 0, ceiling 1
    boxes = []
    for _ in range(n_boxes):
        size = rng.uniform(0.3, 2.0, 3)
        size[2] = min(size[2], 2.2)
        lo = rng.uniform([0.3, 0.3, 0.0], L - size - [0.3, 0.3, 0.5])
        lo[2] = 0.0                                         # on the floor
        lo = np.round(lo * 64) / 64
        hi = np.round((lo + size) * 64) / 64
        boxes.append((lo, hi))
        meshes.append(box(lo, hi, int(rng.integers(0, 4))))
    v, t, m = merge(*meshes)
    fs = fs_of(h, 1.0)
    alpha = rng.uniform(0.05, 0.8, (4, 3))
    coef = np.stack([design_octave_cascade_np(fs, a) for a in alpha])
    pts = _free_points(rng, L, boxes, 5, 0.6)
    sig = diff_gaussian(steps, 8.0)[None, :]
    return Scene("furnished_room", v, t, m, np.arange(4, dtype=np.uint8), h, 0.0, 1.0, 16, steps, 4, 3, coef,
                 pts[:1], sig, pts[1:], seed=seed)


def large_hall(seed: int = 3, steps: int = 4000, size=(1024, 768, 512), h: float = 1.0 / 64.0) -> Scene:
    rng = np.random.default_rng(seed)
    L = np.array(size, np.float64) * h
    v, t, m = box((0, 0, 0), L, [0, 0, 0, 0, 1, 0])        # floor material 1, the rest 0
    fs = fs_of(h, 1.0)
    alpha = rng.uniform(0.05, 0.8, (2, 3))
    coef = np.stack([design_octave_cascade_np(fs, a) for a in alpha])
    src = _interior_points(rng, (0, 0, 0), L, 1, 1.0)
    rcv = _interior_points(rng, (0, 0, 0), L, 8, 1.0)
    sig = gaussian(steps, 8.0)[None, :]
    return Scene("large_hall", v, t, m, np.array([0, 1], np.uint8), h, 0.0, 1.0, 1, steps, 2, 3, coef,
                 src, sig, rcv, seed=seed)


def batched(seed: int = 5, steps: int = 3000, n_sources: int = 64, n_rooms: int = 16, room: int = 256,
            size_range=(96, 320), h: float = 1.0 / 64.0) -> list[Scene]:
    """The batched workload: n_sources seeded source positions in one room of
    room^3 voxels (one simulation per source) plus n_rooms rooms whose voxel
    counts lie between size_range[0]^3 and size_range[1]^3 with seeded aspect
    ratios and 1-4 materials (3-section cascades), each with one source and
    one receiver."""
    rng = np.random.default_rng(seed)
    fs = fs_of(h, 1.0)
    out = []
    L = np.full(3, room * h)
    v, t, m = box((0, 0, 0), L, [0, 0, 0, 0, 1, 1])
    alpha = rng.uniform(0.05, 0.8, (2, 3))
    coef = np.stack([design_octave_cascade_np(fs, a) for a in alpha])
    rcv = _interior_points(rng, (0, 0, 0), L, 1, 0.5)
    srcs = _interior_points(rng, (0, 0, 0), L, n_sources, 0.5)
    sig = diff_gaussian(steps, 8.0)[None, :]
    for k in range(n_sources):
        out.append(Scene(f"batch_src{k}", v, t, m, np.array([0, 1], np.uint8), h, 0.0, 1.0, 1, steps, 2, 3, coef,
                         srcs[k:k + 1], sig, rcv, seed=seed))
    for k in range(n_rooms):
        side = rng.uniform(size_range[0], size_range[1])
        aspect = rng.uniform(0.6, 1.6, 3)
        aspect /= np.cbrt(aspect.prod())
        dims = np.clip(np.round(side * aspect / 8) * 8, 32, 512)
        L = dims * h
        nm = int(rng.integers(1, 5))
        v, t, m = box((0, 0, 0), L, rng.integers(0, nm, 6))
        alpha = rng.uniform(0.05, 0.8, (nm, 3))
        coef = np.stack([design_octave_cascade_np(fs, a) for a in alpha])
        src = _interior_points(rng, (0, 0, 0), L, 1, 0.3)
        rc = _interior_points(rng, (0, 0, 0), L, 1, 0.3)
        out.append(Scene(f"batch_room{k}", v, t, m, np.arange(nm, dtype=np.uint8), h, 0.0, 1.0, 1, steps, nm, 3,
                         coef, src, sig, rc, seed=seed))
    return out


def inverse_design(seed: int = 6, steps: int = 4000, size=(128, 128, 96), h: float = 1.0 / 64.0,
                   n_materials: int = 6, n_sections: int = 2, n_receivers: int = 4):
    """The inverse-design workload: a room of `size` voxels whose six faces
    carry six materials of two sections each (12 coefficient sets, the
    learnable parameters), one source, four receivers.  Returns
    (scene with the hidden coefficients, initial-guess coefficients)."""
    rng = np.random.default_rng(seed)
    L = np.array(size, np.float64) * h
    v, t, m = box((0, 0, 0), L, np.arange(6) % n_materials)
    fs = fs_of(h, 1.0)
    hidden = np.stack([design_octave_cascade_np(fs, a)[:n_sections] for a in rng.uniform(0.1, 0.7, (n_materials, 3))])
    guess = np.stack([design_octave_cascade_np(fs, a)[:n_sections] for a in rng.uniform(0.1, 0.7, (n_materials, 3))])
    src = _interior_points(rng, (0, 0, 0), L, 1, 0.3)
    rcv = _interior_points(rng, (0, 0, 0), L, n_receivers, 0.3)
    sig = diff_gaussian(steps, 6.0)[None, :]
    sc = Scene("inverse_design", v, t, m, np.arange(n_materials, dtype=np.uint8), h, 0.0, 1.0, 1, steps,
               n_materials, n_sections, hidden, src, sig, rcv, seed=seed)
    return sc, guess


def reference_room(seed: int = 4, steps: int = 300, size=(48, 40, 32), h: float = 0.05) -> Scene:
    """The reference's configuration on a small grid: material 0 walls,
    material 1 a speaker box (hard source), default filter and constants."""
    rng = np.random.default_rng(seed)
    L = np.array(size, np.float64) * h
    room = box((0, 0, 0), L, 0)
    c = rng.uniform(L * 0.3, L * 0.5)
    spk = box(c, c + 2.2 * h, 1)
    v, t, m = merge(room, spk)
    rcv = _interior_points(rng, (0, 0, 0), L, 3, 4 * h)
    return Scene("reference_room", v, t, m, np.array([0, 0xFE], np.uint8), h, 0.1, 0.5, 1, steps, 1, 1, None,
                 np.zeros((0, 3)), None, rcv, seed=seed)


def _free_points(rng, L, boxes, n, margin):
    out = []
    while len(out) < n:
        p = rng.uniform(margin, L - margin)
        if all(not np.all((p > lo - margin) & (p < hi + margin)) for lo, hi in boxes):
            out.append(p)
    return np.array(out)


# ---- small helpers that only need numpy (the library has the same designs) ----

def fs_of(h: float, courant: float, c: float = 343.0) -> float:
    """1/dt in double as the filter design sees it (simulator.cpp:940-952)."""
    dt = float(np.float32(courant)) * float(np.float32(h)) / (c * np.sqrt(3.0))
    return 1.0 / dt


# absorber designs used by the scene builders: the library's by default; a
# caller that must not load the library (the benchmark's CPU arm) installs
# other implementations of the same designs with `designs`
_DESIGNS = {}


@contextlib.contextmanager
def designs(first_order, octave_cascade):
    """Build scenes with these absorber designs (callables with the
    signatures of design_first_order_np / design_octave_cascade_np) instead
    of the library's, inside the `with` block."""
    old = dict(_DESIGNS)
    _DESIGNS.update(first_order=first_order, octave_cascade=octave_cascade)
    try:
        yield
    finally:
        _DESIGNS.clear()
        _DESIGNS.update(old)


def design_first_order_np(fs: float, reflection: float, fc: float) -> np.ndarray:
    if "first_order" in _DESIGNS:
        return np.asarray(_DESIGNS["first_order"](fs, reflection, fc), np.float64)
    from . import capi
    return capi.design_first_order(fs, reflection, fc)


def design_octave_cascade_np(fs: float, alpha) -> np.ndarray:
    if "octave_cascade" in _DESIGNS:
        return np.asarray(_DESIGNS["octave_cascade"](fs, alpha), np.float64)
    from . import capi
    return capi.design_octave_cascade(fs, alpha)


def voxel_index(pos, bbox_min, h, shape) -> np.ndarray:
    """World position -> reference voxel index (Simulator::getGridIdxFromVecPos,
    simulator.h:32-35: toVoxel then truncation)."""
    nx, ny, nz = shape
    p = np.atleast_2d(np.asarray(pos, np.float32))
    v = (p - np.asarray(bbox_min, np.float32)) / np.float32(h)
    ix = v.astype(np.int64)
    ix = np.clip(ix, 1, np.array([nx - 2, ny - 2, nz - 2]))
    return (ix[:, 2] * ny + ix[:, 1]) * nx + ix[:, 0]


def boundary_form(sc: Scene) -> int:
    """The reference's explicit boundary correction for the reference
    Courant number (0.5/sqrt 3); the centered form at the 3D limit, where a
    thick explicit damping layer diverges."""
    return 0 if sc.courant <= 0.5 else 1


def build_simulation(sc: Scene, *, storage: int = 0, device: int = 0, boundary_k: float = 0.0,
                     form: int | None = None, storage_scale: float = 0.0, steps: int | None = None):
    """Create, voxelise, classify and configure a Simulation for a scene and
    start it from rest.  Returns (sim, info dict)."""
    from . import capi
    p = capi.default_params(device=device, courant=sc.courant, cell_size=sc.cell_size, bbox_nudge=sc.nudge,
                            sponge_width=sc.sponge_width, storage=storage, storage_scale=storage_scale,
                            boundary_k=boundary_k,
                            boundary_form=boundary_form(sc) if form is None else form)
    sim = capi.Simulation(p)
    sim.set_material_roles(sc.roles)
    sim.set_mesh(sc.verts, sc.tris, sc.tri_mat)
    sim.classify()
    g = sim.info()
    shape = (int(g.nx), int(g.ny), int(g.nz))
    bmin = np.array(list(g.bbox_min), np.float32)
    if sc.coef64 is not None:
        sim.set_filters(sc.coef64.astype(np.float32), n_sections=sc.n_sections)
    if sc.hard is not None:
        sim.set_hard_source(sc.hard)
    src = voxel_index(sc.src_pos, bmin, g.cell_size, shape) if len(sc.src_pos) else np.zeros(0, np.uint64)
    rcv = voxel_index(sc.rcv_pos, bmin, g.cell_size, shape) if len(sc.rcv_pos) else np.zeros(0, np.uint64)
    if src.size:
        sim.set_sources(src, sc.src_sig)
    sim.set_receivers(rcv)
    sim.start(sc.steps if steps is None else steps)
    return sim, dict(shape=shape, bmin=bmin, src=src, rcv=rcv, info=g)


def build_slabs(sc: Scene, parts: int, *, storage: int = 0, device: int = 0, storage_scale: float = 0.0,
                steps: int | None = None, form: int | None = None, voxelise: str = "slab"):
    """The scene's grid split into `parts` z-slabs, one handle each on
    `device`, each configured like build_simulation with the sources and
    receivers it owns.  voxelise="slab": every slab voxelises its own planes
    of the mesh (virs_set_mesh_slab); "whole": the mesh is voxelised once
    and every slab gets its planes of the flags and wall materials
    (virs_set_grid_slab).  Returns ([(sim, z_lo, z_hi,
    receivers_owned_mask)], info dict)."""
    from . import capi, slabs
    p = capi.default_params(device=device, courant=sc.courant, cell_size=sc.cell_size, bbox_nudge=sc.nudge,
                            sponge_width=sc.sponge_width, storage=storage, storage_scale=storage_scale,
                            boundary_form=boundary_form(sc) if form is None else form)
    sims = []
    if voxelise == "whole":
        with capi.Simulation(p) as whole:
            whole.set_material_roles(sc.roles)
            whole.set_mesh(sc.verts, sc.tris, sc.tri_mat)
            flags, wmat, g = whole.flags(), whole.wall_materials(), whole.info()
        shape = (int(g.nx), int(g.ny), int(g.nz))
        for r in range(parts):
            s = capi.Simulation(p)
            slabs.setup_slab(s, shape, g.cell_size, flags, wmat, r, parts, sc.sponge_width)
            sims.append(s)
    else:
        for r in range(parts):
            s = capi.Simulation(p)
            s.set_material_roles(sc.roles)
            s.set_mesh_slab(sc.verts, sc.tris, sc.tri_mat, r, parts)
            sims.append(s)
        g = sims[0].info()
        shape = (int(g.nx), int(g.ny), sims[0].slab_info()[2])
    bmin = np.array(list(g.bbox_min), np.float32)
    src = voxel_index(sc.src_pos, bmin, g.cell_size, shape) if len(sc.src_pos) else np.zeros(0, np.uint64)
    rcv = voxel_index(sc.rcv_pos, bmin, g.cell_size, shape) if len(sc.rcv_pos) else np.zeros(0, np.uint64)
    out = []
    for s in sims:
        z_lo, z_hi, _ = s.slab_info()
        s.classify()
        if sc.coef64 is not None:
            s.set_filters(sc.coef64.astype(np.float32), n_sections=sc.n_sections)
        if sc.hard is not None:
            s.set_hard_source(sc.hard)
        own_s, loc_s = slabs.local_index(src, shape, z_lo, z_hi)
        if loc_s.size:
            s.set_sources(loc_s, np.asarray(sc.src_sig, np.float32).reshape(src.size, -1)[own_s])
        own_r, loc_r = slabs.local_index(rcv, shape, z_lo, z_hi)
        s.set_receivers(loc_r)
        s.start(sc.steps if steps is None else steps)
        out.append((s, z_lo, z_hi, own_r))
    return out, dict(shape=shape, bmin=bmin, src=src, rcv=rcv, info=g)
