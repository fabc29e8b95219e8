"""The CPU oracle, pinned against the reference's own code and against
known answers.  CPU only."""
import numpy as np
import pytest

import oracle
from helpers import oracle_grid, oracle_scene, rel_l2
from virs_b200 import scenes


def _ref(fast=False):
    L = oracle.ref_host(fast)
    if L is None:
        pytest.skip("reference-built checkers (oracle/_ref) not built")
    return L


# ---- pinned against the reference's own sources --------------------------------

def _sat_cases(n, seed):
    rng = np.random.default_rng(seed)
    lo = np.floor(rng.uniform(0, 4, (n, 3))).astype(np.float32)
    boxes = np.concatenate([lo, lo + 1], 1).astype(np.float32)
    tris = (lo[:, None, :] + rng.uniform(-1.5, 2.5, (n, 3, 3))).reshape(-1, 9).astype(np.float32)
    k = n // 3
    tris[:k] = np.round(tris[:k] * 2) / 2          # vertices on half-voxel lattice: touching cases
    tris[k:2 * k] = np.round(tris[k:2 * k])        # on the voxel lattice: faces lying on box faces
    return tris, boxes


@pytest.mark.parametrize("fast", [False, True])
def test_sat_matches_reference_build(fast):
    L = _ref(fast)
    tris, boxes = _sat_cases(60000, 7)
    ref = np.zeros(len(tris), np.uint8)
    L.ref_sat_batch(tris, boxes, len(tris), ref)
    mine = np.array([oracle.sat(t[:3], t[3:6], t[6:], b[:3], b[3:]) for t, b in zip(tris, boxes)], np.uint8)
    assert 0.1 < ref.mean() < 0.9
    assert np.array_equal(ref, mine)


@pytest.mark.parametrize("h", [343 / 88200, 0.025, 1 / 64, 0.05])
@pytest.mark.parametrize("courant", [0.5, 1.0])
def test_highpass_matches_reference_build(h, courant):
    L = _ref()
    h = float(np.float32(h))
    fs = oracle.filter_fs(h, 343.0, courant)
    for fc, q in [(440.0, 0.1), (100.0, 0.7), (5000.0, 2.0)]:
        mine = oracle.rbj_highpass_ref(fs, fc, q)
        ref = np.zeros(5, np.float32)
        L.ref_highpass(fs, fc, q, 1.0, ref)
        assert mine.view(np.uint32).tolist() == ref.view(np.uint32).tolist()
        mine = oracle.rbj_lowpass_ref(fs, fc, q)
        L.ref_lowpass(fs, fc, q, 1.0, ref)
        assert mine.view(np.uint32).tolist() == ref.view(np.uint32).tolist()


def test_highpass_fast_math_build_close():
    L = _ref(True)
    fs = oracle.filter_fs(float(np.float32(343 / 88200)))
    mine = oracle.rbj_highpass_ref(fs, 440.0, 0.1)
    ref = np.zeros(5, np.float32)
    L.ref_highpass(fs, 440.0, 0.1, 1.0, ref)
    assert np.max(np.abs(mine.view(np.int32) - ref.view(np.int32))) <= 2


# ---- known answers -----------------------------------------------------------------

def test_reference_constants():
    h = float(np.float32(343.0 / 88200.0))
    dt, c2dt2, inv_h2, K = oracle.step_constants(h, 343.0, 0.5)
    assert abs(float(c2dt2) * float(inv_h2) - 1 / 12) < 1e-6           # lambda^2 = 1/12
    assert abs(float(K) - 0.95 * 0.5 / np.sqrt(3)) < 1e-6
    assert abs(oracle.filter_fs(h) - 305533.755) < 1e-2                 # 1/dt in double


def test_bbox_keeps_flt_min_start():
    v = np.array([[-3, -2, -1], [-1, -0.5, -0.25]], np.float32)
    lo, hi = oracle.bbox(v, 0.0)
    assert lo.tolist() == [-3, -2, -1]
    assert np.all(hi == np.float32(np.finfo(np.float32).tiny))          # numeric_limits<float>::min()


def test_grid_dims_of_configs():
    for L, h, want in [((4.0, 3.0, 2.5), 0.025, (160, 120, 100)), ((8.0, 6.0, 3.0), 1 / 64, (512, 384, 192)),
                       ((16.0, 12.0, 8.0), 1 / 64, (1024, 768, 512))]:
        v, _, _ = scenes.box((0, 0, 0), L, 0)
        lo, hi = oracle.bbox(v, 0.0)
        assert oracle.dims(lo, hi, float(np.float32(h))) == want


def test_sponge_rule_is_face_neighbourhood_at_width_1():
    """sponge_kernel.cu:50: minDist2 < N*N+1 with N = 1 admits d2 = 1 only."""
    shape = (9, 9, 9)
    f = np.zeros(9 ** 3, np.uint8)
    f[(4 * 9 + 4) * 9 + 4] = 1
    out, _, bd2 = oracle.classify(shape, 1, f)
    got = np.flatnonzero(out == 2)
    c = (4 * 9 + 4) * 9 + 4
    assert sorted(got.tolist()) == sorted([c + 1, c - 1, c + 9, c - 9, c + 81, c - 81])
    out2, _, bd2 = oracle.classify(shape, 2, f)
    assert np.count_nonzero(out2 == 2) == 32                            # |{d: 0 < |d|^2 <= 4}| = 32
    assert set(bd2[out2 == 2].tolist()) == {1, 2, 3, 4}


def test_sponge_nearest_material_tie_break():
    """Nearest wall wins; on equal d2 the first in (dz, dy, dx) order."""
    shape = (9, 9, 9)
    f = np.zeros(9 ** 3, np.uint8)
    wm = np.zeros_like(f)
    c = (4 * 9 + 4) * 9 + 4
    f[c - 2] = 1; wm[c - 2] = 5        # dx = -2
    f[c + 2] = 1; wm[c + 2] = 6        # dx = +2 (same d2, later in scan order)
    f[c - 162] = 1; wm[c - 162] = 7    # dz = -2 (same d2, earliest in scan order)
    out, bm, bd2 = oracle.classify(shape, 2, f, wm)
    assert out[c] == 2 and bd2[c] == 4 and bm[c] == 7


def _classify_cube_scan(shape, W, flags, wmat):
    """sponge_kernel.cu:8-62 generalised to width W as written: each
    interior air voxel scans its whole cube in (dz, dy, dx) order and keeps
    the first smallest squared distance to a wall voxel."""
    nx, ny, nz = shape
    f = flags.reshape(nz, ny, nx)
    out = f.copy()
    bm = np.zeros_like(f)
    bd = np.zeros(f.shape, np.uint16)
    for z in range(1, nz - 1):
        for y in range(1, ny - 1):
            for x in range(1, nx - 1):
                if f[z, y, x] != 0:
                    continue
                best, where = 1 << 30, None
                for dz in range(-W, W + 1):
                    for dy in range(-W, W + 1):
                        for dx in range(-W, W + 1):
                            zz, yy, xx = z + dz, y + dy, x + dx
                            if 0 <= zz < nz and 0 <= yy < ny and 0 <= xx < nx and f[zz, yy, xx] == 1:
                                d2 = dx * dx + dy * dy + dz * dz
                                if d2 < best:
                                    best, where = d2, (zz, yy, xx)
                if best < W * W + 1:
                    out[z, y, x] = 2
                    bm[z, y, x] = wmat.reshape(f.shape)[where]
                    bd[z, y, x] = best
                else:
                    out[z, y, x] = 0
    return out.reshape(-1), bm.reshape(-1), bd.reshape(-1)


@pytest.mark.parametrize("seed", range(4))
def test_classification_equals_cube_scan(seed):
    """The oracle's classification (the cube scan with rows reduced to
    their nearest wall voxels) against the literal cube scan: flags,
    nearest-wall materials and distances on random small grids."""
    rng = np.random.default_rng(seed)
    shape = tuple(int(v) for v in rng.integers(4, 14, 3))
    W = int(rng.integers(1, 5))
    n = int(np.prod(shape))
    flags = np.zeros(n, np.uint8)
    flags[rng.random(n) < rng.uniform(0.02, 0.15)] = 1
    flags[rng.random(n) < 0.02] = 3
    wmat = rng.integers(0, 4, n).astype(np.uint8)
    got = oracle.classify(shape, W, flags, wmat)
    want = _classify_cube_scan(shape, W, flags, wmat)
    for a, b in zip(got, want):
        assert np.array_equal(np.asarray(a).reshape(-1), np.asarray(b).reshape(-1).astype(np.asarray(a).dtype))


def test_boundary_list_sorted_interior():
    sc = scenes.reference_room()
    g = oracle_grid(sc)
    b = g["bidx"].astype(np.int64)
    assert np.all(np.diff(b) > 0)
    nx, ny, nz = g["shape"]
    x, y, z = b % nx, (b // nx) % ny, b // (nx * ny)
    assert x.min() >= 1 and y.min() >= 1 and z.min() >= 1
    assert x.max() <= nx - 2 and y.max() <= ny - 2 and z.max() <= nz - 2
    assert np.all(g["flags"][b] == 2)


def _closed_box(n=(14, 12, 10)):
    nx, ny, nz = n
    f = np.zeros(nx * ny * nz, np.uint8).reshape(nz, ny, nx)
    f[0, :, :] = f[-1, :, :] = 1
    f[:, 0, :] = f[:, -1, :] = 1
    f[:, :, 0] = f[:, :, -1] = 1
    return n, f.reshape(-1)


@pytest.mark.parametrize("courant", [0.5, 1.0])
def test_energy_conserved_without_boundary_filter(courant):
    shape, f = _closed_box()
    flags, _, _ = oracle.classify(shape, 1, f)
    bidx = oracle.boundary_list(shape, flags)
    dt, c2dt2, inv_h2, K = oracle.step_constants(0.05, 343.0, courant)
    rng = np.random.default_rng(0)
    p = rng.standard_normal(flags.size).astype(np.float32) * (flags != 1)
    p = p.reshape(shape[::-1])
    p[0], p[-1], p[:, 0], p[:, -1], p[:, :, 0], p[:, :, -1] = 0, 0, 0, 0, 0, 0
    p = np.ascontiguousarray(p.reshape(-1))
    pp = p.copy()
    sc = oracle.Scene(shape, flags, bidx, np.zeros(bidx.size, np.uint8), np.ones(bidx.size, np.float32),
                      np.zeros(5, np.float32), 1, consts=(c2dt2, inv_h2, K), gain=0.0)
    lam2 = float(c2dt2) * float(inv_h2)
    e0 = oracle.energy(shape, flags, p, pp, lam2)
    st = np.zeros(bidx.size * 4 + 1, np.float32)
    sc.run(200, state=(p, pp, st))
    e1 = oracle.energy(shape, flags, p, pp, lam2)
    assert abs(e1 - e0) / e0 < 1e-4


def test_impulse_symmetry():
    """A centred impulse in a symmetric closed box stays mirror-symmetric."""
    shape, f = _closed_box((15, 13, 11))
    nx, ny, nz = shape
    flags, _, _ = oracle.classify(shape, 1, f)
    bidx = oracle.boundary_list(shape, flags)
    dt, c2dt2, inv_h2, K = oracle.step_constants(0.05, 343.0, 0.5)
    fs = oracle.filter_fs(0.05)
    c = oracle.rbj_highpass_ref(fs, 440, 0.1)
    sc = oracle.Scene(shape, flags, bidx, np.zeros(bidx.size, np.uint8), np.ones(bidx.size, np.float32), c, 1,
                      consts=(c2dt2, inv_h2, K))
    p = np.zeros(flags.size, np.float32)
    p[((nz // 2) * ny + ny // 2) * nx + nx // 2] = 1.0
    pp = p.copy()
    sc.run(60, state=(p, pp, np.zeros(bidx.size * 4 + 1, np.float32)))
    v = p.reshape(nz, ny, nx)
    assert np.abs(v).max() > 0
    # x-mirror swaps the first two summands only (a + b = b + a): exact;
    # y / z mirrors reorder a floating-point sum: equal to rounding
    assert np.array_equal(v, np.flip(v, axis=2))
    for ax in (0, 1):
        assert np.max(np.abs(v - np.flip(v, axis=ax))) <= 1e-5 * np.abs(v).max()


def test_hand_checked_update():
    """One interior step on a 5x5x5 grid against the formula written out."""
    shape = (5, 5, 5)
    flags = np.zeros(125, np.uint8)
    flags[(2 * 5 + 2) * 5 + 3] = 1                      # a wall at +x of the centre
    rng = np.random.default_rng(3)
    p = rng.uniform(-1, 1, 125).astype(np.float32)
    pp = rng.uniform(-1, 1, 125).astype(np.float32)
    c2dt2, inv_h2 = np.float32(0.25), np.float32(0.5)
    sc = oracle.Scene(shape, flags, np.zeros(0, np.uint32), None, None, np.zeros(5, np.float32), 1,
                      consts=(c2dt2, inv_h2, np.float32(0)))
    p0, pp0 = p.copy(), pp.copy()
    st = np.zeros(1, np.float32)
    sc.run(1, state=(p, pp, st))
    i = (2 * 5 + 2) * 5 + 2
    ce = p0[i]
    nb = [ce, p0[i - 1], p0[i + 5], p0[i - 5], p0[i + 25], p0[i - 25]]   # +x is the wall: mirrored
    s = np.float32(nb[0])
    for v in nb[1:]:
        s = np.float32(s + v)
    lap = np.float32(np.float64(s) - 6.0 * np.float64(ce))  # fma: one rounding
    lap = np.float32(lap * inv_h2)
    want = np.float32(np.float64(np.float32(2 * ce - pp0[i])) + np.float64(c2dt2) * np.float64(lap))
    assert p[i] == want
    assert p[(2 * 5 + 2) * 5 + 3] == 0.0                 # the wall voxel is zeroed
    assert np.all(p.reshape(5, 5, 5)[0] == 0)           # border never written (was p_next = 0)


def test_fp32_close_to_fp64_reference_room():
    sc = scenes.reference_room(steps=200)
    g = oracle_grid(sc)
    osc = oracle_scene(sc, g)
    a = osc.run(sc.steps)
    b = osc.run(sc.steps, f64=True)
    assert np.isfinite(a).all()
    assert rel_l2(a, b) < 1e-5


@pytest.mark.parametrize("form,courant", [(0, 0.5), (1, 1.0)])
def test_fp64_adjoint_matches_finite_differences(form, courant):
    """Gradients of an IR loss w.r.t. filter coefficients and source samples
    from the FP64 adjoint (checkpoints every 16 steps) against central
    differences with h = 1e-3, Richardson-extrapolated (h and h/2) to remove
    the O(h^2) truncation of the strongly non-linear denominator terms."""
    import dataclasses
    sc, _ = scenes.inverse_design(steps=120, size=(20, 18, 14), h=0.05, n_materials=3)
    sc = dataclasses.replace(sc, courant=courant)
    if form == 0:
        sc = dataclasses.replace(sc, coef64=sc.coef64)
    g = oracle_grid(sc)
    osc = oracle_scene(sc, g)
    osc.form = form
    target = osc.run64(sc.steps) * 0.9 + 0.01

    def loss():
        ir = osc.run64(sc.steps)
        return np.sum((ir - target) ** 2) / ir.size, ir

    _, ir = loss()
    gc, gs = osc.adjoint64(sc.steps, 2 * (ir - target) / ir.size, every=16)

    def fd(setv, base, h):
        setv(base + h); lp, _ = loss()
        setv(base - h); lm, _ = loss()
        setv(base)
        return (lp - lm) / (2 * h)

    for (m, s, j) in [(0, 0, 0), (1, 1, 3), (2, 0, 4), (0, 1, 1), (2, 1, 2)]:
        k = (m * osc.n_sections + s) * 5 + j
        base = osc.coef64[k]

        def setv(v, k=k):
            osc.coef64[k] = v

        d1, d2 = fd(setv, base, 1e-3), fd(setv, base, 5e-4)
        rich = (4 * d2 - d1) / 3
        assert abs(rich - gc[m, s, j]) <= 1e-4 * abs(gc[m, s, j]) + 1e-14, (m, s, j, rich, gc[m, s, j])
    for (s, n) in [(0, 10), (0, 60)]:
        base = float(osc.src_sig[s, n])
        h = np.float32(1e-3)

        def setv(v, s=s, n=n):
            osc.src_sig[s, n] = v

        setv(np.float32(base) + h); lp, _ = loss()
        up = float(osc.src_sig[s, n])
        setv(np.float32(base) - h); lm, _ = loss()
        dn = float(osc.src_sig[s, n])
        setv(np.float32(base))
        assert abs((lp - lm) / (up - dn) - gs[s, n]) <= 1e-6 * abs(gs[s, n])


def test_storage_rounding_matches_ieee_conversions():
    """The oracle's 16-bit storage rounding: FP16 as IEEE binary16 (ties to
    even, subnormals, overflow to infinity), BF16 as the top half of the
    FP32 word rounded to nearest even."""
    rng = np.random.default_rng(0)
    x = rng.standard_normal(100000).astype(np.float32) * np.float32(10.0) ** rng.integers(-12, 6, 100000).astype(np.float32)
    x = np.concatenate([x, np.array([65504, 65519.99, 65520, -65520, 6.1e-5, 6.0e-5, 3e-8, 2.98e-8, 1e-9, 0.0, -0.0,
                                     np.inf, -np.inf], np.float32)]).astype(np.float32)
    with np.errstate(over="ignore"):
        want16 = x.astype(np.float16).astype(np.float32)
    assert np.array_equal(oracle.round16(x, 1).view(np.uint32), want16.view(np.uint32))
    u = x.view(np.uint32).astype(np.uint64)
    wantb = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    assert np.array_equal(oracle.round16(x, 2).view(np.uint32), wantb)


def test_oracle_absorber_designs_equal_the_library():
    """The oracle's FP64 absorber designs (used by the benchmark's CPU arm
    instead of the library's) equal the library's bit for bit."""
    from virs_b200 import capi
    rng = np.random.default_rng(3)
    for _ in range(100):
        fs = rng.uniform(2e4, 4e5)
        a = rng.uniform(0.05, 1.0, 3)
        got = oracle.design_octave_cascade(fs, a)
        want = np.asarray(capi.design_octave_cascade(fs, a), np.float64).reshape(3, 5)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        r, fc = rng.uniform(-0.9, 0.99), rng.uniform(50.0, fs / 2.5)
        got = oracle.design_first_order(fs, r, fc)
        want = np.asarray(capi.design_first_order(fs, r, fc), np.float64)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("storage", [1, 2])
def test_stochastic_rounding_is_unbiased_and_exact_on_representable_values(storage):
    """The library's stochastic rounding (restated in the oracle): every
    result is one of the two neighbouring 16-bit values, values already
    representable never move, and over all 2^16 random words the mean of
    the results is the value itself (exactly, in double)."""
    rng = np.random.default_rng(7)
    r = np.arange(65536, dtype=np.uint32)
    xs = rng.normal(0, 50, 40).astype(np.float32)
    if storage == 1:
        xs = np.concatenate([xs, np.float32([1e-3, -3.5e-4, 60000.0])])
    for x in xs:
        y = oracle.sr16(np.full(65536, x, np.float32), storage, r)
        vals = sorted({float(v) for v in y})
        assert len(vals) <= 2
        near = float(oracle.round16(np.float32([x]), storage)[0])
        assert near in vals
        assert abs(float(np.mean(y.astype(np.float64))) - float(x)) <= 1e-12 * abs(float(x)) + 1e-30
        rep = oracle.round16(np.float32([x]), storage)
        assert np.array_equal(oracle.sr16(np.full(65536, rep[0], np.float32), storage, r), np.full(65536, rep[0]))
