/*
 * virs_oracle.c -- CPU restatement of the VIRS room-acoustics FDTD path.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  This library is the checker that the
 * CUDA implementation under virs_b200/ is compared against.  Only tests/,
 * __graft_entry__.smoke() and the cpu_baseline / reference legs of bench.py
 * load it; the product library never links or calls it.
 *
 * What it restates (paths relative to the Snipet/VIRS source tree):
 *   - triangle/box SAT test            src/simulator/simulator.cpp:45-141
 *   - bounding box + grid sizing       src/simulator/simulator.cpp:288-329
 *   - toVoxel                          src/simulator/simulator.h:39-45
 *   - triangle sweep -> flags 1 / 3    src/simulator/simulator.cpp:396-452
 *   - boundary ("sponge") marking      src/simulator/sponge_kernel.cu:8-62
 *   - neighbour normals bitmask        src/simulator/simulator.cpp:480-531
 *   - boundary index list              src/simulator/simulator.cpp:572-605
 *   - RBJ high-pass design             src/simulator/biquad.cpp:24-43
 *   - step constants                   src/simulator/simulator_gpu.cu:195-198, simulator.cpp:940-957
 *   - interior leapfrog update         src/simulator/simulator_gpu.cu:38-103
 *   - boundary biquad update           src/simulator/simulator_gpu.cu:105-150
 *   - source value, rotation, receiver src/simulator/simulator_gpu.cu:214-218, 292-300
 *
 * Extensions with no reference counterpart (their definition lives here and
 * the CUDA path must agree with it):
 *   - sponge width W (the reference hard-codes N = 1, sponge_kernel.cu:5):
 *     air voxels with a wall voxel at squared distance d2 <= W*W become
 *     boundary voxels; W = 1 is exactly the reference rule;
 *   - per-boundary-voxel material: material of the nearest wall voxel, ties
 *     broken by the reference's scan order (dz, dy, dx ascending, strict <);
 *   - per-material cascades of S biquad sections (series form; S = 1 is the
 *     reference's single section);
 *   - sponge weight w(d2) = ((W + 1 - sqrt(d2)) / W)^2 on the boundary
 *     correction (w = 1 whenever W = 1);
 *   - additive ("soft") point sources with per-step signals, R receivers.
 *
 * Floating point: the FP32 run follows the reference CUDA build's numerics:
 * nvcc --use_fast_math flushes subnormals (FTZ) and contracts a*b+c into one
 * fused multiply-add.  This file compiles with -ffp-contract=off, writes every
 * fused operation explicitly with fmaf(), and sets the x86 FTZ/DAZ bits in
 * every worker thread for the FP32 run.  The boundary correction is evaluated
 * in double exactly as the reference does (simulator_gpu.cu:148, the double
 * literals 0.1 and 0.9 promote the expression).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>
#include <pmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VO_API __attribute__((visibility("default")))

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------ */
/* threading / FTZ                                                           */
/* ------------------------------------------------------------------------ */

static int g_threads = 0; /* 0 = OpenMP default */

VO_API void vo_set_threads(int n) { g_threads = n; }

VO_API int vo_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

static void ftz_on(void)
{
    _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
    _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
}

static void ftz_off(void)
{
    _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_OFF);
    _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_OFF);
}

/* ------------------------------------------------------------------------ */
/* geometry                                                                  */
/* ------------------------------------------------------------------------ */

typedef struct { float x, y, z; } v3;

static v3 v3sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3 v3abs(v3 a) { v3 r = {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; return r; }
static float mn3(float a, float b, float c) { float m = a; if (b < m) m = b; if (c < m) m = c; return m; }
static float mx3(float a, float b, float c) { float m = a; if (m < b) m = b; if (m < c) m = c; return m; }

/* simulator.cpp:73-86 -- note the projection always uses the .y and .z
 * components of the vertices, whatever the edge/axis pair; kept as written. */
static int axis_test(float a, float b, float fa, float fb, v3 p0, v3 p1, v3 p2, float ex, float ey)
{
    float p0p = a * p0.y - b * p0.z;
    float p1p = a * p1.y - b * p1.z;
    float p2p = a * p2.y - b * p2.z;
    float minp = mn3(p0p, p1p, p2p);
    float maxp = mx3(p0p, p1p, p2p);
    float rad = fa * ey + fb * ex;
    return !(minp > rad || maxp < -rad);
}

/* simulator.cpp:45-141 */
static int sat(v3 v0w, v3 v1w, v3 v2w, v3 bmin, v3 bmax)
{
    v3 c = {(bmin.x + bmax.x) * 0.5f, (bmin.y + bmax.y) * 0.5f, (bmin.z + bmax.z) * 0.5f};
    v3 e = {(bmax.x - bmin.x) * 0.5f, (bmax.y - bmin.y) * 0.5f, (bmax.z - bmin.z) * 0.5f};
    v3 v0 = v3sub(v0w, c), v1 = v3sub(v1w, c), v2 = v3sub(v2w, c);
    v3 f0 = v3sub(v1, v0), f1 = v3sub(v2, v1), f2 = v3sub(v0, v2);
    v3 a0 = v3abs(f0), a1 = v3abs(f1), a2 = v3abs(f2);

    if (!axis_test(f0.z, f0.y, a0.z, a0.y, v0, v1, v2, e.y, e.z)) return 0;
    if (!axis_test(f0.z, f0.x, a0.z, a0.x, v0, v1, v2, e.x, e.z)) return 0;
    if (!axis_test(f0.y, f0.x, a0.y, a0.x, v0, v1, v2, e.x, e.y)) return 0;
    if (!axis_test(f1.z, f1.y, a1.z, a1.y, v0, v1, v2, e.y, e.z)) return 0;
    if (!axis_test(f1.z, f1.x, a1.z, a1.x, v0, v1, v2, e.x, e.z)) return 0;
    if (!axis_test(f1.y, f1.x, a1.y, a1.x, v0, v1, v2, e.x, e.y)) return 0;
    if (!axis_test(f2.z, f2.y, a2.z, a2.y, v0, v1, v2, e.y, e.z)) return 0;
    if (!axis_test(f2.z, f2.x, a2.z, a2.x, v0, v1, v2, e.x, e.z)) return 0;
    if (!axis_test(f2.y, f2.x, a2.y, a2.x, v0, v1, v2, e.x, e.y)) return 0;

    float lo = mn3(v0.x, v1.x, v2.x), hi = mx3(v0.x, v1.x, v2.x);
    if (lo > e.x || hi < -e.x) return 0;
    lo = mn3(v0.y, v1.y, v2.y); hi = mx3(v0.y, v1.y, v2.y);
    if (lo > e.y || hi < -e.y) return 0;
    lo = mn3(v0.z, v1.z, v2.z); hi = mx3(v0.z, v1.z, v2.z);
    if (lo > e.z || hi < -e.z) return 0;

    v3 n = {f0.y * f1.z - f0.z * f1.y, f0.z * f1.x - f0.x * f1.z, f0.x * f1.y - f0.y * f1.x};
    float d = -(n.x * v0.x + n.y * v0.y + n.z * v0.z);
    float r = e.x * fabsf(n.x) + e.y * fabsf(n.y) + e.z * fabsf(n.z);
    if (fabsf(d) > r) return 0;
    return 1;
}

VO_API int vo_sat(const float *v0, const float *v1, const float *v2, const float *bmin, const float *bmax)
{
    v3 a = {v0[0], v0[1], v0[2]}, b = {v1[0], v1[1], v1[2]}, c = {v2[0], v2[1], v2[2]};
    v3 lo = {bmin[0], bmin[1], bmin[2]}, hi = {bmax[0], bmax[1], bmax[2]};
    return sat(a, b, c, lo, hi);
}

/* simulator.cpp:288-310.  The max corner starts at FLT_MIN (the smallest
 * positive normal float, numeric_limits<float>::min()), not -FLT_MAX, so an
 * axis whose vertices are all negative keeps max = FLT_MIN; reproduced. */
VO_API void vo_bbox(const float *verts, uint64_t nverts, float nudge, float *bmin, float *bmax)
{
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
    for (uint64_t i = 0; i < nverts; ++i)
        for (int a = 0; a < 3; ++a) {
            float v = verts[3 * i + a];
            if (v < lo[a]) lo[a] = v;
            if (hi[a] < v) hi[a] = v;
        }
    for (int a = 0; a < 3; ++a) {
        bmin[a] = lo[a] - nudge;
        bmax[a] = hi[a] + nudge;
    }
}

/* simulator.cpp:321-329: span * (1/h), truncated to size_t. */
VO_API void vo_dims(const float *bmin, const float *bmax, float h, uint64_t *dims)
{
    float nvm = 1.f / h;
    for (int a = 0; a < 3; ++a) {
        float span = bmax[a] - bmin[a];
        float s = span * nvm;
        dims[a] = s > 0.f ? (uint64_t)s : 0;
    }
}

/* simulator.h:39-45 */
static v3 to_voxel(v3 p, const float *bmin, float h)
{
    v3 r = {(p.x - bmin[0]) / h, (p.y - bmin[1]) / h, (p.z - bmin[2]) / h};
    return r;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Roles of OBJ material ids.  roles[m] for m < nroles:
 *   0xFF = ignored, 0xFE = source ("speaker", flag 3), k < 0xFE = wall with
 *   absorber material k (flag 1).  Ids outside the table (including -1, a
 *   face with no usemtl) are ignored.  The reference mapping is
 *   {0: wall, 1: speaker} (simulator.cpp:439-449). */
#define VO_ROLE_IGNORE 0xFF
#define VO_ROLE_SOURCE 0xFE

/* simulator.cpp:396-452.  tris: ntri * 9 floats (world coordinates). */
VO_API int vo_voxelize(const float *tris, const int32_t *tri_mat, uint64_t ntri,
                       const uint8_t *roles, uint64_t nroles, float h, const float *bmin,
                       uint64_t nx, uint64_t ny, uint64_t nz, uint8_t *flags, uint8_t *wall_mat)
{
    if (nx == 0 || ny == 0 || nz == 0) return -1;
    for (uint64_t t = 0; t < ntri; ++t) {
        int m = tri_mat[t];
        uint8_t role = (m >= 0 && (uint64_t)m < nroles) ? roles[m] : VO_ROLE_IGNORE;
        const float *q = tris + 9 * t;
        v3 w0 = {q[0], q[1], q[2]}, w1 = {q[3], q[4], q[5]}, w2 = {q[6], q[7], q[8]};
        v3 g0 = to_voxel(w0, bmin, h), g1 = to_voxel(w1, bmin, h), g2 = to_voxel(w2, bmin, h);
        int ix0 = clampi((int)floorf(mn3(g0.x, g1.x, g2.x)), 0, (int)nx - 1);
        int iy0 = clampi((int)floorf(mn3(g0.y, g1.y, g2.y)), 0, (int)ny - 1);
        int iz0 = clampi((int)floorf(mn3(g0.z, g1.z, g2.z)), 0, (int)nz - 1);
        int ix1 = clampi((int)ceilf(mx3(g0.x, g1.x, g2.x)), 0, (int)nx - 1);
        int iy1 = clampi((int)ceilf(mx3(g0.y, g1.y, g2.y)), 0, (int)ny - 1);
        int iz1 = clampi((int)ceilf(mx3(g0.z, g1.z, g2.z)), 0, (int)nz - 1);
        for (int k = iz0; k <= iz1; ++k)
            for (int j = iy0; j <= iy1; ++j)
                for (int i = ix0; i <= ix1; ++i) {
                    v3 lo = {(float)i, (float)j, (float)k};
                    v3 hi = {(float)i + 1.f, (float)j + 1.f, (float)k + 1.f};
                    if (!sat(g0, g1, g2, lo, hi)) continue;
                    uint64_t idx = ((uint64_t)k * ny + (uint64_t)j) * nx + (uint64_t)i;
                    if (role == VO_ROLE_SOURCE) {
                        flags[idx] = 3;
                    } else if (role != VO_ROLE_IGNORE) {
                        flags[idx] = 1;
                        if (wall_mat) wall_mat[idx] = role;
                    }
                }
    }
    return 0;
}

/* sponge_kernel.cu:8-62 generalised to width W.  Interior voxels with flag 0
 * scan the cube [-W, W]^3 for wall voxels (flag 1); the smallest squared
 * distance d2 wins (first in dz, dy, dx order on ties, as the reference's
 * strict "<" keeps the first).  d2 < W*W + 1 marks the voxel 2.  Voxels with
 * flag != 0 are copied; the domain border is left as it was.  bmat / bd2
 * receive, per voxel, the nearest wall's material and d2 (0 elsewhere). */
VO_API void vo_classify(uint64_t nx, uint64_t ny, uint64_t nz, int W, const uint8_t *flags_in,
                        const uint8_t *wall_mat, uint8_t *flags_out, uint8_t *bmat, uint16_t *bd2)
{
    const uint64_t n = nx * ny * nz;
    if (flags_out != flags_in) memcpy(flags_out, flags_in, n);
    if (bmat) memset(bmat, 0, n);
    if (bd2) memset(bd2, 0, n * sizeof(uint16_t));
    const int lim = W * W + 1;
    /* Per row of the cube only the wall voxels nearest to x on either side
     * can win: d2 = dx^2 + dy^2 + dz^2 grows with |dx| within a row, and of
     * two at the same |dx| the scan (dx ascending, strict <) keeps the one
     * at -|dx|.  So the row's candidate is its nearest wall at or left of x
     * unless the nearest at or right of x is strictly closer, and rows are
     * then compared in the cube's (dz, dy) order with the same strict <:
     * the same winner as scanning every voxel of the cube.  lft / rgt hold,
     * per voxel, the x of the nearest wall voxel at or before / at or after
     * it in its row (-1 / nx when there is none). */
    int32_t *lft = malloc(n * sizeof(int32_t)), *rgt = malloc(n * sizeof(int32_t));
    if (!lft || !rgt) { free(lft); free(rgt); return; }
#pragma omp parallel for schedule(static) num_threads(vo_get_threads())
    for (int64_t r = 0; r < (int64_t)(ny * nz); ++r) {
        const uint8_t *row = flags_in + (uint64_t)r * nx;
        int32_t *L = lft + (uint64_t)r * nx, *R = rgt + (uint64_t)r * nx;
        int32_t last = -1;
        for (uint64_t x = 0; x < nx; ++x) { if (row[x] == 1) last = (int32_t)x; L[x] = last; }
        last = (int32_t)nx;
        for (uint64_t x = nx; x-- > 0;) { if (row[x] == 1) last = (int32_t)x; R[x] = last; }
    }
    /* one output row at a time: the cube's rows in (dz, dy) order, each
     * compared with every voxel's best so far (the per-voxel order of the
     * scan is unchanged, the loops are only interchanged) */
#pragma omp parallel num_threads(vo_get_threads())
    {
        int *best = malloc(nx * sizeof(int));
        uint64_t *bestn = malloc(nx * sizeof(uint64_t));
#pragma omp for schedule(dynamic, 1)
        for (int64_t zy = 0; zy < (int64_t)(ny * nz); ++zy) {
            const int64_t z = zy / (int64_t)ny, y = zy % (int64_t)ny;
            if (!best || !bestn || z < 1 || z >= (int64_t)nz - 1 || y < 1 || y >= (int64_t)ny - 1) continue;
            for (uint64_t x = 0; x < nx; ++x) best[x] = 1 << 30;
            for (int dz = -W; dz <= W; ++dz) {
                const int64_t zz = z + dz;
                if (zz < 0 || zz >= (int64_t)nz) continue;
                for (int dy = -W; dy <= W; ++dy) {
                    const int64_t yy = y + dy;
                    if (yy < 0 || yy >= (int64_t)ny) continue;
                    const uint64_t r = (uint64_t)zz * ny + (uint64_t)yy;
                    const int32_t *L = lft + r * nx, *R = rgt + r * nx;
                    const int e = dy * dy + dz * dz;
                    for (int64_t x = 1; x < (int64_t)nx - 1; ++x) {
                        const int64_t l = L[x], g = R[x];
                        int64_t dx;
                        if (l >= 0 && x - l <= W && (g >= (int64_t)nx || g - x > W || x - l <= g - x))
                            dx = l - x;
                        else if (g < (int64_t)nx && g - x <= W)
                            dx = g - x;
                        else
                            continue;                       /* no wall voxel within [x-W, x+W] */
                        const int d2 = (int)(dx * dx) + e;
                        if (d2 < best[x]) {
                            best[x] = d2;
                            bestn[x] = r * nx + (uint64_t)(x + dx);
                        }
                    }
                }
            }
            for (int64_t x = 1; x < (int64_t)nx - 1; ++x) {
                const uint64_t id = ((uint64_t)z * ny + (uint64_t)y) * nx + (uint64_t)x;
                if (flags_in[id] != 0) continue;
                if (best[x] < lim) {
                    flags_out[id] = 2;
                    if (bmat) bmat[id] = wall_mat ? wall_mat[bestn[x]] : 0;
                    if (bd2) bd2[id] = (uint16_t)best[x];
                } else {
                    flags_out[id] = 0;
                }
            }
        }
        free(best);
        free(bestn);
    }
    free(lft);
    free(rgt);
}

/* simulator.cpp:480-531: bit set for each of the 6 neighbours whose flag is 0
 * (+x 1, -x 2, +y 4, -y 8, +z 16, -z 32), interior voxels only. */
VO_API void vo_normals(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t *flags, uint8_t *normals)
{
    memset(normals, 0, nx * ny * nz);
    const uint64_t sy = nx, sz = nx * ny;
    for (uint64_t z = 1; z + 1 < nz; ++z)
        for (uint64_t y = 1; y + 1 < ny; ++y)
            for (uint64_t x = 1; x + 1 < nx; ++x) {
                uint64_t i = z * sz + y * sy + x;
                uint8_t c = 0;
                if (flags[i - 1] == 0) c |= 2;
                if (flags[i + 1] == 0) c |= 1;
                if (flags[i - sy] == 0) c |= 8;
                if (flags[i + sy] == 0) c |= 4;
                if (flags[i - sz] == 0) c |= 32;
                if (flags[i + sz] == 0) c |= 16;
                normals[i] = c;
            }
}

/* simulator.cpp:572-605: ascending indices of interior voxels with flag 2.
 * Returns the count; out may be NULL (counting pass). */
VO_API uint64_t vo_boundary_list(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t *flags, uint32_t *out)
{
    uint64_t k = 0;
    for (uint64_t z = 1; z + 1 < nz; ++z)
        for (uint64_t y = 1; y + 1 < ny; ++y)
            for (uint64_t x = 1; x + 1 < nx; ++x) {
                uint64_t i = (z * ny + y) * nx + x;
                if (flags[i] == 2) {
                    if (out) out[k] = (uint32_t)i;
                    ++k;
                }
            }
    return k;
}

/* ------------------------------------------------------------------------ */
/* constants and coefficient design                                          */
/* ------------------------------------------------------------------------ */

/* simulator_gpu.cu:195-198 with the Courant factor made a parameter
 * (reference: 0.5):  dt = s*h/(c*sqrt(3)), c2dt2 = c*c*dt*dt, inv_h2 = 1/h^2;
 * simulator_gpu.cu:147: K = (c*dt)/h * 0.95 (evaluated here in IEEE single;
 * the reference evaluates it on the device). */
VO_API void vo_step_constants(float h, float c, float courant, float *out4)
{
    float dt = courant * h / (c * sqrtf(3.f));
    float c2dt2 = c * c * dt * dt;
    float inv_h2 = 1.f / (h * h);
    float K = (c * dt) / h * 0.95f;
    out4[0] = dt;
    out4[1] = c2dt2;
    out4[2] = inv_h2;
    out4[3] = K;
}

/* simulator.cpp:940-952: the host computes dt again in double and the filter
 * sample rate as 1/dt, narrowed to float at the call of the design. */
VO_API double vo_filter_fs(float h, double c, double courant)
{
    double hd = (double)h;
    double dt = courant * hd / (c * sqrt(3.0));
    return 1.f / dt;
}

/* biquad.cpp:24-43 (RBJ high-pass), with the same float/double promotions:
 * 2.f * M_PI is double, so omega is computed in double and stored to float;
 * sin/cos of a float argument call the double functions. */
VO_API void vo_rbj_highpass_ref(float fs, float cutoff, float q, float gain, float *out5)
{
    float omega = 2.f * M_PI * cutoff / fs;
    float alpha = sin(omega) / (2.f * q);
    float a0 = 1.f + alpha;
    float b0 = (1.f + cos(omega)) / 2.f / a0;
    float b1 = -(1.f + cos(omega)) / a0;
    float b2 = b0;
    float a1 = -2.f * cos(omega) / a0;
    float a2 = (1.f - alpha) / a0;
    b0 *= gain; b1 *= gain; b2 *= gain;
    out5[0] = b0; out5[1] = b1; out5[2] = b2; out5[3] = a1; out5[4] = a2;
}

/* biquad.cpp:3-22 (RBJ low-pass) with the same promotions. */
VO_API void vo_rbj_lowpass_ref(float fs, float cutoff, float q, float gain, float *out5)
{
    float omega = 2.f * M_PI * cutoff / fs;
    float alpha = sin(omega) / (2.f * q);
    float a0 = 1.f + alpha;
    float b0 = (1.f - cos(omega)) / 2.f / a0;
    float b1 = (1.f - cos(omega)) / a0;
    float b2 = b0;
    float a1 = -2.f * cos(omega) / a0;
    float a2 = (1.f - alpha) / a0;
    b0 *= gain; b1 *= gain; b2 *= gain;
    out5[0] = b0; out5[1] = b1; out5[2] = b2; out5[3] = a1; out5[4] = a2;
}

/* sponge weight w(d2) = ((W + 1 - sqrt(d2)) / W)^2, 1 at d2 = 1. */
VO_API float vo_sponge_weight(int W, int d2)
{
    double d = sqrt((double)d2);
    double t = ((double)W + 1.0 - d) / (double)W;
    if (t < 0.0) t = 0.0;
    return (float)(t * t);
}

/* ------------------------------------------------------------------------ */
/* time stepping                                                             */
/* ------------------------------------------------------------------------ */

typedef struct vo_run_args {
    uint64_t nx, ny, nz;
    const uint8_t *flags;          /* classified flags, N bytes            */
    uint64_t nb;                   /* boundary voxels                      */
    const uint32_t *bidx;          /* [nb] ascending indices               */
    const uint8_t *bmat;           /* [nb] material of each boundary voxel */
    const float *bw;               /* [nb] sponge weight (NULL = all 1)    */
    uint32_t n_materials;
    uint32_t n_sections;
    const float *coef32;           /* [M][S][5] b0 b1 b2 a1 a2             */
    const double *coef64;          /* same, FP64 run                       */
    float c2dt2, inv_h2, K;        /* FP32 run constants                   */
    double c2dt2_d, inv_h2_d, K_d; /* FP64 run constants                   */
    double mix_y, mix_d;           /* 0.1, 0.9 (simulator_gpu.cu:148)      */
    double gain;                   /* (double)0.4f                         */
    int32_t form;                  /* 0 reference (explicit), 1 centered   */
    const float *hard;             /* flag-3 value per step                */
    uint64_t n_hard;
    uint32_t n_src;
    const uint64_t *src_idx;
    const float *src_sig;          /* [n_src][sig_len]                     */
    uint64_t sig_len;
    uint32_t n_rcv;
    const uint64_t *rcv_idx;
    uint64_t steps;
    uint64_t step0;                /* index of the first step (source time)*/
    uint64_t ir_stride;            /* row stride of ir (>= steps)          */
    float *ir;                     /* [n_rcv][ir_stride], written at [r][n]*/
    void *p;                       /* in/out p^n      (float or double)    */
    void *pprev;                   /* in/out p^{n-1}                       */
    void *state;                   /* in/out [nb][S][4]                    */
    double *ir64;                  /* FP64 run: IR in double (may be NULL) */
    int32_t storage;               /* FP32 run: 0 FP32 fields, 1 FP16, 2 BF16 */
    float scale;                   /* 16-bit storage: fields hold scale * p  */
    int32_t rigid;                 /* FP32 run: rigid-wall update of boundary voxels */
    float l2;                      /* (c dt / h)^2 of that update            */
    const uint8_t *normals;        /* air-neighbour mask per voxel           */
    int32_t rounding;              /* 16-bit storage: 0 to nearest, 1 stochastic */
    uint64_t sr_base;              /* its key offset (a slab's first padded voxel) */
} vo_run_args;

/* 16-bit field storage, as the GPU path stores it: every value written to
 * a field is rounded to the nearest FP16 / BF16 value (ties to even; FP16
 * keeps its subnormals, overflow gives infinity); loads are exact.  The
 * fields hold scale * p with a power-of-two scale, so the FP32 arithmetic
 * on them is the same as on p, scaled. */
static inline float vo_round_bf16(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) {            /* inf stays, NaN quiet */
        if (u & 0x007fffffu) u |= 0x00400000u;
        u &= 0xffff0000u;
    } else {
        u += 0x7fffu + ((u >> 16) & 1u);
        u &= 0xffff0000u;
    }
    memcpy(&x, &u, 4);
    return x;
}

static inline float vo_round_f16(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    const uint32_t sign = u & 0x80000000u, a = u & 0x7fffffffu;
    if (a >= 0x7f800000u) return x;                       /* inf, NaN */
    if (a >= 0x477ff000u) {                               /* >= 65520: rounds to inf */
        u = sign | 0x7f800000u;
        memcpy(&x, &u, 4);
        return x;
    }
    if (a < 0x38800000u) {                                /* below 2^-14: FP16 subnormal */
        float m;
        memcpy(&m, &a, 4);
        const float q = nearbyintf(m * 16777216.0f);      /* multiples of 2^-24, ties to even */
        float r = q * (1.0f / 16777216.0f);
        uint32_t v;
        memcpy(&v, &r, 4);
        v |= sign;
        memcpy(&x, &v, 4);
        return x;
    }
    uint32_t v = a + 0xfffu + ((a >> 13) & 1u);           /* 23 -> 10 mantissa bits */
    v = (v & ~0x1fffu) | sign;
    memcpy(&x, &v, 4);
    return x;
}

/* The FP64 absorber designs of the library (no reference counterpart):
 * the definitions the benchmark's CPU arm designs its cascades with, so that
 * it needs no part of the library.
 * First order: bilinear transform, prewarped at fc, of G wc / (s + wc) with
 * G = (1 - R) / (1 + R); out5 = {b0, b1, b2, a1, a2}. */
VO_API void vo_design_first_order(double fs, double reflection, double fc, double *out5)
{
    const double g = (1.0 - reflection) / (1.0 + reflection);
    const double k = tan(M_PI * fc / fs);
    out5[0] = g * k / (1.0 + k);
    out5[1] = g * k / (1.0 + k);
    out5[2] = 0.0;
    out5[3] = (k - 1.0) / (k + 1.0);
    out5[4] = 0.0;
}

static void vo_norm5(double *o, double b0, double b1, double b2, double a0, double a1, double a2)
{
    o[0] = b0 / a0; o[1] = b1 / a0; o[2] = b2 / a0; o[3] = a1 / a0; o[4] = a2 / a0;
}

/* Octave cascade from absorption alpha[0..2] at 250, 1000 and 4000 Hz: band
 * gains G_b = (1 - R_b) / (1 + R_b), R_b = sqrt(1 - alpha_b), as an RBJ low
 * shelf (G_0 below 250 Hz), a peaking section (G_1 at 1 kHz, Q = 1/sqrt 2)
 * and a high shelf (G_2 above 4 kHz), shelf slope 1; out15 = 3 x out5. */
VO_API void vo_design_octave_cascade(double fs, const double *alpha, double *out15)
{
    const double f[3] = {250.0, 1000.0, 4000.0};
    double G[3];
    for (int b = 0; b < 3; ++b) {
        const double R = sqrt(1.0 - alpha[b]);
        G[b] = (1.0 - R) / (1.0 + R);
    }
    {
        const double A = sqrt(G[0]);
        const double w = 2.0 * M_PI * f[0] / fs, cw = cos(w), al = sin(w) / 2.0 * sqrt(2.0);
        const double sA = 2.0 * sqrt(A) * al;
        vo_norm5(out15, A * ((A + 1) - (A - 1) * cw + sA), 2 * A * ((A - 1) - (A + 1) * cw),
                 A * ((A + 1) - (A - 1) * cw - sA), (A + 1) + (A - 1) * cw + sA, -2 * ((A - 1) + (A + 1) * cw),
                 (A + 1) + (A - 1) * cw - sA);
    }
    {
        const double A = sqrt(G[1]);
        const double w = 2.0 * M_PI * f[1] / fs, cw = cos(w), al = sin(w) / (2.0 / sqrt(2.0));
        vo_norm5(out15 + 5, 1 + al * A, -2 * cw, 1 - al * A, 1 + al / A, -2 * cw, 1 - al / A);
    }
    {
        const double A = sqrt(G[2]);
        const double w = 2.0 * M_PI * f[2] / fs, cw = cos(w), al = sin(w) / 2.0 * sqrt(2.0);
        const double sA = 2.0 * sqrt(A) * al;
        vo_norm5(out15 + 10, A * ((A + 1) + (A - 1) * cw + sA), -2 * A * ((A - 1) + (A + 1) * cw),
                 A * ((A + 1) + (A - 1) * cw - sA), (A + 1) - (A - 1) * cw + sA, 2 * ((A - 1) - (A + 1) * cw),
                 (A + 1) - (A - 1) * cw - sA);
    }
}

/* initSphereKernel (src/simulator/init_sphere.cu:4-25), one loop iteration
 * per thread of its 3D grid: every voxel (x, y, z) of the nx*ny*nz field
 * whose integer squared distance to (cx, cy, cz) is at most r^2 (the
 * launcher passes radius * radius, init_sphere.cu:44) takes `pressure`;
 * with zero_outside every other voxel takes 0, else it keeps its value.
 * Distances are formed from unsigned differences as the kernel does. */
VO_API void vo_init_sphere(float *p, uint64_t nx, uint64_t ny, uint64_t nz, uint64_t cx, uint64_t cy, uint64_t cz,
                           uint64_t radius, float pressure, int zero_outside)
{
    const uint64_t r2 = radius * radius;
    for (uint64_t z = 0; z < nz; ++z)
        for (uint64_t y = 0; y < ny; ++y)
            for (uint64_t x = 0; x < nx; ++x) {
                const uint64_t dx = x > cx ? x - cx : cx - x;
                const uint64_t dy = y > cy ? y - cy : cy - y;
                const uint64_t dz = z > cz ? z - cz : cz - z;
                const uint64_t i = (z * ny + y) * nx + x;
                if (dx * dx + dy * dy + dz * dz <= r2) p[i] = pressure;
                else if (zero_outside) p[i] = 0.f;
            }
}

/* Stochastic rounding of the 16-bit stores, as the library defines it: a
 * value is rounded up in magnitude with the probability of its distance
 * from the value below, using 16 random bits that are a pure function of
 * (voxel, step, phase):
 *   s = mix32(2 step + phase + 0x9e3779b9), w = mix32(((pos + base) >> 1) ^ s),
 *   bits = w & 0xffff for an even pos + base, w >> 16 for an odd one,
 * with pos the voxel's position in the library's padded layout (rows of
 * ceil(nx / 32) * 32 voxels) and phase 0 for the step's store of p^{n+1}
 * (interior, boundary, hard source) and 1 for the soft-source addition.
 * mix32 is the "lowbias32" integer hash (Chris Wellons, hash-prospector).
 * The bits are added below the kept bits of the FP32 pattern, which is then
 * truncated; FP16 values below 2^-14 or of 65504 and more in magnitude, and
 * non-finite values, round to nearest. */
static inline uint32_t vo_mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

static inline uint32_t vo_sr_key(uint64_t step, uint32_t phase)
{
    return vo_mix32((uint32_t)(2u * (uint32_t)step + phase + 0x9e3779b9u));
}

static inline uint32_t vo_sr_bits(uint64_t pos, uint32_t key)
{
    const uint32_t w = vo_mix32((uint32_t)(pos >> 1) ^ key);
    return (pos & 1u) ? (w >> 16) : (w & 0xffffu);
}

static inline float vo_sr16(float x, int storage, uint32_t r16)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    const uint32_t a = u & 0x7fffffffu;
    if (storage == 2) {
        if (a >= 0x7f7f0000u) return vo_round_bf16(x);
        u = (u + r16) & 0xffff0000u;
    } else {
        if (a < 0x38800000u || a >= 0x477fe000u) return vo_round_f16(x);
        u = (u + (r16 & 0x1fffu)) & ~0x1fffu;
    }
    memcpy(&x, &u, 4);
    return x;
}

/* the stochastic rounding on its own (tests): out[i] = in[i] rounded with
 * the random bits r16[i] */
VO_API void vo_sr16_array(const float *in, float *out, uint64_t n, int32_t storage, const uint32_t *r16)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = vo_sr16(in[i], storage, r16[i]);
}

/* padded position of reference index i (rows of px voxels), plus the key offset */
static inline uint64_t vo_padded(const vo_run_args *a, uint64_t i)
{
    const uint64_t px = (a->nx + 31) / 32 * 32, row = i / a->nx;
    return row * px + (i - row * a->nx) + a->sr_base;
}

/* the storage rounding on its own (tests) */
VO_API void vo_round16(const float *in, float *out, uint64_t n, int32_t storage)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = storage == 1 ? vo_round_f16(in[i]) : storage == 2 ? vo_round_bf16(in[i]) : in[i];
}

static void vo_round_field(float *f, uint64_t n, int storage)
{
    if (storage == 0) return;
#pragma omp parallel for num_threads(vo_get_threads()) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) f[i] = storage == 1 ? vo_round_f16(f[i]) : vo_round_bf16(f[i]);
}

/* the step's store of p^{n+1} rounded stochastically (phase 0) */
static void vo_sr_field(const vo_run_args *a, float *f, uint64_t n, uint64_t step)
{
    const uint32_t key = vo_sr_key(step, 0);
#pragma omp parallel for num_threads(vo_get_threads()) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) f[i] = vo_sr16(f[i], a->storage, vo_sr_bits(vo_padded(a, (uint64_t)i), key));
}

static inline float vsel(const uint8_t *fl, const float *p, uint64_t n, float c)
{
    return fl[n] == 1 ? c : p[n];
}

/* simulator_gpu.cu:38-103 -- one thread per interior voxel in the
 * reference; here a z-parallel loop (the reference CPU step's structure,
 * simulator_cpu.cpp:66).  FP32 with FTZ. */
static void interior_f32(const vo_run_args *a, const float *pc, const float *pp, float *pn, float hard)
{
    const uint64_t nx = a->nx, ny = a->ny, nz = a->nz, sy = nx, sz = nx * ny;
    const float c2dt2 = a->c2dt2, inv_h2 = a->inv_h2;
    const uint8_t *fl = a->flags;
#pragma omp parallel num_threads(vo_get_threads())
    {
        ftz_on();
#pragma omp for schedule(static)
        for (int64_t z = 1; z < (int64_t)nz - 1; ++z)
            for (uint64_t y = 1; y + 1 < ny; ++y) {
                const uint64_t row = (uint64_t)z * sz + y * sy;
                for (uint64_t x = 1; x + 1 < nx; ++x) {
                    const uint64_t i = row + x;
                    const uint8_t f = fl[i];
                    if (f == 1) { pn[i] = 0.f; continue; }
                    if (f == 3) { pn[i] = hard; continue; }
                    if (f != 0 && f != 2) continue;
                    const float c = pc[i];
                    float s = vsel(fl, pc, i + 1, c);
                    s = s + vsel(fl, pc, i - 1, c);
                    s = s + vsel(fl, pc, i + sy, c);
                    s = s + vsel(fl, pc, i - sy, c);
                    s = s + vsel(fl, pc, i + sz, c);
                    s = s + vsel(fl, pc, i - sz, c);
                    const float lap = fmaf(-6.f, c, s) * inv_h2;
                    const float t = 2.f * c - pp[i];
                    pn[i] = fmaf(c2dt2, lap, t);
                }
            }
        ftz_off();
    }
}

/* simulator_gpu.cu:105-150 with S sections in series and per-voxel
 * materials; FP32 recursion, double correction. */
static void boundary_f32(const vo_run_args *a, const float *pc, const float *pp, float *pn, float *st)
{
    const uint32_t S = a->n_sections;
    const double K = (double)a->K, my = a->mix_y, md = a->mix_d, g = a->gain;
#pragma omp parallel num_threads(vo_get_threads())
    {
        ftz_on();
#pragma omp for schedule(static)
        for (int64_t b = 0; b < (int64_t)a->nb; ++b) {
            const uint64_t i = a->bidx[b];
            const float d = pc[i] - pp[i];
            float in = d;
            const float *k = a->coef32 + (uint64_t)a->bmat[b] * S * 5;
            float *s = st + (uint64_t)b * S * 4;
            for (uint32_t q = 0; q < S; ++q, k += 5, s += 4) {
                /* nvcc fuses the first two products as fma(b0, in, b1*s0):
                 * found against the reference build's own kernels */
                float y = fmaf(k[0], in, k[1] * s[0]);
                y = fmaf(k[2], s[1], y);
                y = fmaf(-k[3], s[2], y);
                y = fmaf(-k[4], s[3], y);
                s[1] = s[0];
                s[0] = in;
                s[3] = s[2];
                s[2] = y;
                in = y;
            }
            const double w = a->bw ? (double)a->bw[b] : 1.0;
            if (a->form == 0) {
                const double t = fma((double)in, my, (double)d * md);
                const double u = ((K * t) * g) * w;
                pn[i] = (float)((double)pn[i] - u);
            } else {
                /* centered damping: the direct term uses (p+ - p-)/2 */
                const double kgw = (K * g) * w;
                const double ac = (kgw * md) * 0.5;
                const double num = ((double)pn[i] - kgw * ((double)in * my)) + ac * (double)pp[i];
                pn[i] = (float)(num / (1.0 + ac));
            }
        }
        ftz_off();
    }
}

/* fdtd_kernel_rigid_walls (simulator_gpu.cu:152-180): a boundary voxel's
 * update from its air neighbours only (the normals mask: neighbour flag 0),
 * p+ = (2 - l2 n) p - p- + sum over the six neighbours, in the order +x,
 * -x, +y, -y, +z, -z, of (l2 * s) * p_nb with s = 1 for an air neighbour
 * and 0 otherwise; it replaces the interior update before the filter
 * correction.  With the contractions of the reference build (found against
 * its own kernel, tests/golden/rigid_room.npz): b1 = fma(-l2, n, 2),
 * p = fma(b1, p, -p-), then fma(l2 * s, p_nb, p) per neighbour. */
static void rigid_f32(const vo_run_args *a, const float *pc, const float *pp, float *pn)
{
    const uint64_t sy = a->nx, sz = a->nx * a->ny;
    const float l2 = a->l2;
#pragma omp parallel num_threads(vo_get_threads())
    {
        ftz_on();
#pragma omp for schedule(static)
        for (int64_t b = 0; b < (int64_t)a->nb; ++b) {
            const uint64_t i = a->bidx[b];
            const uint8_t m = a->normals[i];
            int nn = 0;
            for (uint8_t v = m; v; v &= (uint8_t)(v - 1)) ++nn;
            const float b1 = fmaf(-l2, (float)nn, 2.f);
            float r = fmaf(b1, pc[i], -pp[i]);
            const uint64_t nb6[6] = {i + 1, i - 1, i + sy, i - sy, i + sz, i - sz};
            for (int k = 0; k < 6; ++k) r = fmaf(l2 * ((m & (1u << k)) ? 1.f : 0.f), pc[nb6[k]], r);
            pn[i] = r;
        }
        ftz_off();
    }
}

static float sig_at(const vo_run_args *a, uint32_t s, uint64_t n)
{
    return n < a->sig_len ? a->src_sig[(uint64_t)s * a->sig_len + n] : 0.f;
}

/* One run of a->steps FP32 steps.  a->p / a->pprev / a->state hold the
 * initial state (NULL = zero) and receive the final one. */
VO_API int vo_run_f32(const vo_run_args *a)
{
    const uint64_t N = a->nx * a->ny * a->nz;
    float *b0 = calloc(N, sizeof(float)), *b1 = calloc(N, sizeof(float)), *b2 = calloc(N, sizeof(float));
    const uint64_t nst = a->nb * a->n_sections * 4;
    float *st = calloc(nst ? nst : 1, sizeof(float));
    if (!b0 || !b1 || !b2 || !st) { free(b0); free(b1); free(b2); free(st); return -1; }
    if (a->p) memcpy(b0, a->p, N * sizeof(float));
    if (a->pprev) memcpy(b1, a->pprev, N * sizeof(float));
    if (a->state) memcpy(st, a->state, nst * sizeof(float));
    float *pc = b0, *pp = b1, *pn = b2;
    const int sto = a->storage;
    const float scale = sto ? a->scale : 1.f, inv_scale = 1.f / scale;
    /* the next buffer starts as the reference's p_next would: it holds the
     * values the kernel never writes (the domain border stays 0). */
    for (uint64_t n = 0; n < a->steps; ++n) {
        const uint64_t sn = a->step0 + n;
        const float hard = sn < a->n_hard ? a->hard[sn] * scale : 0.f;
        interior_f32(a, pc, pp, pn, hard);
        if (a->nb && a->rigid) rigid_f32(a, pc, pp, pn);
        if (a->nb) boundary_f32(a, pc, pp, pn, st);
        const int sr = sto && a->rounding == 1;
        if (sr) vo_sr_field(a, pn, N, sn);
        else vo_round_field(pn, N, sto);
        for (uint32_t s = 0; s < a->n_src; ++s) {
            const uint64_t i = a->src_idx[s];
            const float v = sig_at(a, s, sn) * scale;   /* scaled on the host, without FTZ */
            ftz_on();
            pn[i] = pn[i] + v;
            ftz_off();
            if (sr) pn[i] = vo_sr16(pn[i], sto, vo_sr_bits(vo_padded(a, i), vo_sr_key(sn, 1)));
            else if (sto) pn[i] = sto == 1 ? vo_round_f16(pn[i]) : vo_round_bf16(pn[i]);
        }
        /* rotation (simulator_gpu.cu:292-293): prev <- curr <- next */
        float *t = pp; pp = pc; pc = pn; pn = t;
        ftz_on();
        for (uint32_t r = 0; r < a->n_rcv; ++r)
            a->ir[(uint64_t)r * a->ir_stride + n] = sto ? pc[a->rcv_idx[r]] * inv_scale : pc[a->rcv_idx[r]];
        ftz_off();
    }
    if (a->p) memcpy(a->p, pc, N * sizeof(float));
    if (a->pprev) memcpy(a->pprev, pp, N * sizeof(float));
    if (a->state) memcpy(a->state, st, nst * sizeof(float));
    free(b0); free(b1); free(b2); free(st);
    return 0;
}

/* One step of the model in double precision (interior, boundary, sources). */
static void f64_step(const vo_run_args *a, const double *pc, const double *pp, double *pn, double *st, uint64_t sn)
{
    const uint64_t nx = a->nx, ny = a->ny, nz = a->nz, sy = nx, sz = nx * ny;
    const uint8_t *fl = a->flags;
    const uint32_t S = a->n_sections;
    const double hard = sn < a->n_hard ? (double)a->hard[sn] : 0.0;
    const double c2dt2 = a->c2dt2_d, inv_h2 = a->inv_h2_d;
#pragma omp parallel for schedule(static) num_threads(vo_get_threads())
    for (int64_t z = 1; z < (int64_t)nz - 1; ++z)
        for (uint64_t y = 1; y + 1 < ny; ++y)
            for (uint64_t x = 1; x + 1 < nx; ++x) {
                const uint64_t i = (uint64_t)z * sz + y * sy + x;
                const uint8_t f = fl[i];
                if (f == 1) { pn[i] = 0.0; continue; }
                if (f == 3) { pn[i] = hard; continue; }
                if (f != 0 && f != 2) continue;
                const double c = pc[i];
                double s = (fl[i + 1] == 1 ? c : pc[i + 1]) + (fl[i - 1] == 1 ? c : pc[i - 1]) +
                           (fl[i + sy] == 1 ? c : pc[i + sy]) + (fl[i - sy] == 1 ? c : pc[i - sy]) +
                           (fl[i + sz] == 1 ? c : pc[i + sz]) + (fl[i - sz] == 1 ? c : pc[i - sz]);
                pn[i] = 2.0 * c - pp[i] + c2dt2 * ((s - 6.0 * c) * inv_h2);
            }
#pragma omp parallel for schedule(static) num_threads(vo_get_threads())
    for (int64_t b = 0; b < (int64_t)a->nb; ++b) {
        const uint64_t i = a->bidx[b];
        const double d = pc[i] - pp[i];
        double in = d;
        const double *k = a->coef64 + (uint64_t)a->bmat[b] * S * 5;
        double *s = st + (uint64_t)b * S * 4;
        for (uint32_t q = 0; q < S; ++q, k += 5, s += 4) {
            double y = k[0] * in + k[1] * s[0] + k[2] * s[1] - k[3] * s[2] - k[4] * s[3];
            s[1] = s[0]; s[0] = in; s[3] = s[2]; s[2] = y; in = y;
        }
        const double w = a->bw ? (double)a->bw[b] : 1.0;
        if (a->form == 0) {
            pn[i] -= a->K_d * (in * a->mix_y + d * a->mix_d) * a->gain * w;
        } else {
            const double kgw = a->K_d * a->gain * w, ac = kgw * a->mix_d * 0.5;
            pn[i] = (pn[i] - kgw * in * a->mix_y + ac * pp[i]) / (1.0 + ac);
        }
    }
    for (uint32_t s = 0; s < a->n_src; ++s) pn[a->src_idx[s]] += (double)sig_at(a, s, sn);
}

/* The same model in double precision: the truth the reduced-precision forms
 * are measured against.  Coefficients come from a->coef64. */
VO_API int vo_run_f64(const vo_run_args *a)
{
    if (a->rigid) return -2; /* the rigid-wall update is an FP32-run option */
    const uint64_t N = a->nx * a->ny * a->nz;
    double *b0 = calloc(N, sizeof(double)), *b1 = calloc(N, sizeof(double)), *b2 = calloc(N, sizeof(double));
    const uint64_t nst = a->nb * a->n_sections * 4;
    double *st = calloc(nst ? nst : 1, sizeof(double));
    if (!b0 || !b1 || !b2 || !st) { free(b0); free(b1); free(b2); free(st); return -1; }
    if (a->p) memcpy(b0, a->p, N * sizeof(double));
    if (a->pprev) memcpy(b1, a->pprev, N * sizeof(double));
    if (a->state) memcpy(st, a->state, nst * sizeof(double));
    double *pc = b0, *pp = b1, *pn = b2;
    for (uint64_t n = 0; n < a->steps; ++n) {
        f64_step(a, pc, pp, pn, st, a->step0 + n);
        double *t = pp; pp = pc; pc = pn; pn = t;
        for (uint32_t r = 0; r < a->n_rcv; ++r) {
            a->ir[(uint64_t)r * a->ir_stride + n] = (float)pc[a->rcv_idx[r]];
            if (a->ir64) a->ir64[(uint64_t)r * a->ir_stride + n] = pc[a->rcv_idx[r]];
        }
    }
    if (a->p) memcpy(a->p, pc, N * sizeof(double));
    if (a->pprev) memcpy(a->pprev, pp, N * sizeof(double));
    if (a->state) memcpy(a->state, st, nst * sizeof(double));
    free(b0); free(b1); free(b2); free(st);
    return 0;
}

/* Reverse-mode gradient of a receiver loss through the FP64 model.
 *
 * Given dL/dIR (dl_dir, [n_rcv][steps]) the adjoint runs the steps backwards.
 * With T the adjoint of p^{n+1} and RR the negated adjoint carried through
 * the q-role of p^n, one reverse step n is:
 *   T[rcv] += dL/dIR_n;  dL/dsig_n = T[src];
 *   F = T, except at boundary voxels where the correction's adjoint acts
 *   (reference form: F = T, ybar = -K g w mix_y T, dbar = -K g w mix_d T;
 *   centered form: F = T/(1+a), ybar = -K g w mix_y T/(1+a), cq = a T/(1+a));
 *   the biquad cascade runs transposed (sections last to first), giving the
 *   coefficient gradients, the state adjoints and dbar += xbar_0;
 *   T' = A F - RR (+ dbar at boundary voxels)   -- the forward leapfrog
 *   RR' = F (+ dbar - cq at boundary voxels).
 * A is symmetric on the updated voxels (walls mirrored, fixed voxels 0), so
 * the interior adjoint is the leapfrog itself.  Forward states are rebuilt
 * from checkpoints taken every `every` steps. */
typedef struct vo_adj_args {
    const vo_run_args *run;       /* forward set-up (FP64 fields used) */
    const double *dl_dir;         /* [n_rcv][steps]                    */
    uint32_t every;               /* checkpoint interval (>= 1)        */
    double *grad_coef;            /* [M][S][5], accumulated            */
    double *grad_sig;             /* [n_src][steps] or NULL            */
} vo_adj_args;

VO_API int vo_adjoint_f64(const vo_adj_args *aa)
{
    const vo_run_args *a = aa->run;
    const uint64_t N = a->nx * a->ny * a->nz, nx = a->nx, ny = a->ny, nz = a->nz, sy = nx, sz = nx * ny;
    const uint64_t steps = a->steps, every = aa->every ? aa->every : 64;
    const uint32_t S = a->n_sections;
    const uint64_t nb = a->nb, nst = nb * S * 4;
    const uint64_t nck = (steps + every - 1) / every;
    const uint8_t *fl = a->flags;
    double *ckp = calloc(nck * N, sizeof(double)), *ckq = calloc(nck * N, sizeof(double));
    double *cks = calloc(nck * (nst ? nst : 1), sizeof(double));
    double *b0 = calloc(N, sizeof(double)), *b1 = calloc(N, sizeof(double)), *b2 = calloc(N, sizeof(double));
    double *st = calloc(nst ? nst : 1, sizeof(double));
    double *segD = calloc(every * (nb ? nb : 1), sizeof(double));
    double *segS = calloc(every * (nst ? nst : 1), sizeof(double));
    double *T = calloc(N, sizeof(double)), *RR = calloc(N, sizeof(double)), *AS = calloc(nst ? nst : 1, sizeof(double));
    double *dbar = calloc(nb ? nb : 1, sizeof(double)), *cqv = calloc(nb ? nb : 1, sizeof(double));
    uint8_t *active = calloc(N, 1);
    int rc = 0;
    if (!ckp || !ckq || !cks || !b0 || !b1 || !b2 || !st || !segD || !segS || !T || !RR || !AS || !dbar || !cqv ||
        !active) { rc = -1; goto done; }
    for (uint64_t z = 1; z + 1 < nz; ++z)
        for (uint64_t y = 1; y + 1 < ny; ++y)
            for (uint64_t x = 1; x + 1 < nx; ++x) {
                const uint64_t i = z * sz + y * sy + x;
                active[i] = fl[i] == 0 || fl[i] == 2;
            }
    {
        /* forward with checkpoints */
        double *pc = b0, *pp = b1, *pn = b2;
        for (uint64_t n = 0; n < steps; ++n) {
            if (n % every == 0) {
                const uint64_t c = n / every;
                memcpy(ckp + c * N, pc, N * sizeof(double));
                memcpy(ckq + c * N, pp, N * sizeof(double));
                if (nst) memcpy(cks + c * nst, st, nst * sizeof(double));
            }
            f64_step(a, pc, pp, pn, st, a->step0 + n);
            double *t = pp; pp = pc; pc = pn; pn = t;
        }
    }
    const double lam2 = a->c2dt2_d * a->inv_h2_d;
    for (int64_t c = (int64_t)nck - 1; c >= 0; --c) {
        const uint64_t n0 = (uint64_t)c * every, n1 = n0 + every < steps ? n0 + every : steps;
        /* rebuild the segment's forward boundary data */
        double *pc = b0, *pp = b1, *pn = b2;
        memcpy(pc, ckp + c * N, N * sizeof(double));
        memcpy(pp, ckq + c * N, N * sizeof(double));
        if (nst) memcpy(st, cks + c * nst, nst * sizeof(double));
        for (uint64_t n = n0; n < n1; ++n) {
            const uint64_t k = n - n0;
            for (uint64_t b = 0; b < nb; ++b) segD[k * nb + b] = pc[a->bidx[b]] - pp[a->bidx[b]];
            if (nst) memcpy(segS + k * nst, st, nst * sizeof(double));
            f64_step(a, pc, pp, pn, st, a->step0 + n);
            double *t = pp; pp = pc; pc = pn; pn = t;
        }
        for (int64_t n = (int64_t)n1 - 1; n >= (int64_t)n0; --n) {
            const uint64_t k = (uint64_t)n - n0;
            for (uint32_t r = 0; r < a->n_rcv; ++r) {
                const uint64_t i = a->rcv_idx[r];
                if (active[i]) T[i] += aa->dl_dir[(uint64_t)r * steps + (uint64_t)n];
            }
            if (aa->grad_sig)
                for (uint32_t s = 0; s < a->n_src; ++s) aa->grad_sig[(uint64_t)s * steps + (uint64_t)n] = T[a->src_idx[s]];
            /* boundary voxels: correction and cascade, transposed */
            for (uint64_t b = 0; b < nb; ++b) {
                const uint64_t i = a->bidx[b];
                const double f = T[i], w = a->bw ? (double)a->bw[b] : 1.0;
                const double kgw = a->K_d * a->gain * w;
                double ybar, db, fr, cq = 0.0;
                if (a->form == 0) {
                    fr = f;
                    ybar = -kgw * a->mix_y * f;
                    db = -kgw * a->mix_d * f;
                } else {
                    const double ac = kgw * a->mix_d * 0.5;
                    fr = f / (1.0 + ac);
                    ybar = -kgw * a->mix_y * fr;
                    db = 0.0;
                    cq = ac * fr;
                }
                /* forward values of the sections at step n */
                const double *k5 = a->coef64 + (uint64_t)a->bmat[b] * S * 5;
                const double *s0 = segS + k * nst + b * S * 4;
                double xin[16];
                double in = segD[k * nb + b];
                for (uint32_t q = 0; q < S; ++q) {
                    const double *kk = k5 + 5 * q, *ss = s0 + 4 * q;
                    xin[q] = in;
                    in = kk[0] * in + kk[1] * ss[0] + kk[2] * ss[1] - kk[3] * ss[2] - kk[4] * ss[3];
                }
                double *as = AS + b * S * 4;
                double *g = aa->grad_coef + (uint64_t)a->bmat[b] * S * 5;
                double yb = ybar;
                for (int32_t q = (int32_t)S - 1; q >= 0; --q) {
                    const double *kk = k5 + 5 * q, *ss = s0 + 4 * q;
                    double *aq = as + 4 * q;
                    const double yt = yb + aq[2];              /* Y1+ = y */
                    g[5 * q + 0] += yt * xin[q];
                    g[5 * q + 1] += yt * ss[0];
                    g[5 * q + 2] += yt * ss[1];
                    g[5 * q + 3] -= yt * ss[2];
                    g[5 * q + 4] -= yt * ss[3];
                    const double xbar = kk[0] * yt + aq[0];    /* X1+ = x */
                    const double x1 = kk[1] * yt + aq[1];      /* X2+ = X1 */
                    const double x2 = kk[2] * yt;
                    const double y1 = -kk[3] * yt + aq[3];     /* Y2+ = Y1 */
                    const double y2 = -kk[4] * yt;
                    aq[0] = x1; aq[1] = x2; aq[2] = y1; aq[3] = y2;
                    yb = xbar;
                }
                db += yb;
                T[i] = fr;
                dbar[b] = db;
                cqv[b] = cq;
            }
            /* T' = A F - RR into RR's buffer; RR' = F (T's buffer) */
#pragma omp parallel for schedule(static) num_threads(vo_get_threads())
            for (int64_t z = 1; z < (int64_t)nz - 1; ++z)
                for (uint64_t y = 1; y + 1 < ny; ++y)
                    for (uint64_t x = 1; x + 1 < nx; ++x) {
                        const uint64_t i = (uint64_t)z * sz + y * sy + x;
                        if (!active[i]) { RR[i] = 0.0; continue; }
                        const double c0 = T[i];
                        double acc = 0.0;
                        const uint64_t nbr[6] = {i + 1, i - 1, i + sy, i - sy, i + sz, i - sz};
                        for (int d = 0; d < 6; ++d)
                            if (fl[nbr[d]] != 1) acc += T[nbr[d]] - c0;
                        RR[i] = 2.0 * c0 - RR[i] + lam2 * acc;
                    }
            for (uint64_t b = 0; b < nb; ++b) {
                const uint64_t i = a->bidx[b];
                RR[i] += dbar[b];
                T[i] += dbar[b] - cqv[b];
            }
            double *t = T; T = RR; RR = t;
        }
    }
done:
    free(ckp); free(ckq); free(cks); free(b0); free(b1); free(b2); free(st); free(segD); free(segS);
    free(T); free(RR); free(AS); free(dbar); free(cqv); free(active);
    return rc;
}

/* Discrete energy of the lossless interior scheme (FP64):
 *   E = sum_{i active} (p_i - q_i)^2
 *     + lambda2 * sum_{links i~j} (p_i - p_j)(q_i - q_j)
 * Active voxels are interior voxels with flag 0/2 (the ones the leapfrog
 * updates).  A link joins an active voxel to a face neighbour that is active
 * (counted once) or held fixed (border voxels and flag-3 voxels, counted
 * once); links to walls (flag 1) carry nothing, which is the mirror rule of
 * simulator_gpu.cu:70-81.  Without boundary filtering and with the fixed
 * voxels at zero, the leapfrog keeps E constant up to rounding.
 * p = p^n, q = p^{n-1}. */
static inline int vo_active(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t *fl, uint64_t j)
{
    const uint64_t x = j % nx, y = (j / nx) % ny, z = j / (nx * ny);
    if (x == 0 || y == 0 || z == 0 || x + 1 >= nx || y + 1 >= ny || z + 1 >= nz) return 0;
    return fl[j] == 0 || fl[j] == 2;
}

VO_API double vo_energy_f32(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t *flags,
                            const float *p, const float *q, double lambda2)
{
    const uint64_t sy = nx, sz = nx * ny;
    double kin = 0.0, pot = 0.0;
#pragma omp parallel for reduction(+ : kin, pot) schedule(static) num_threads(vo_get_threads())
    for (int64_t z = 1; z < (int64_t)nz - 1; ++z)
        for (uint64_t y = 1; y + 1 < ny; ++y)
            for (uint64_t x = 1; x + 1 < nx; ++x) {
                const uint64_t i = (uint64_t)z * sz + y * sy + x;
                if (!vo_active(nx, ny, nz, flags, i)) continue;
                const double d = (double)p[i] - (double)q[i];
                kin += d * d;
                const uint64_t fwd[3] = {i + 1, i + sy, i + sz};
                const uint64_t bwd[3] = {i - 1, i - sy, i - sz};
                for (int a = 0; a < 3; ++a) {
                    uint64_t j = fwd[a];
                    if (flags[j] != 1)
                        pot += ((double)p[i] - (double)p[j]) * ((double)q[i] - (double)q[j]);
                    j = bwd[a];
                    if (flags[j] != 1 && !vo_active(nx, ny, nz, flags, j))
                        pot += ((double)p[i] - (double)p[j]) * ((double)q[i] - (double)q[j]);
                }
            }
    return kin + lambda2 * pot;
}

/* ------------------------------------------------------------------------ */
/* IR post-processing: anti-alias cascade, resampling, normalisation          */
/* ------------------------------------------------------------------------ */

typedef struct { double re, im; } vo_cplx;

static int vo_cmp_imag(const void *a, const void *b)
{
    const double x = ((const vo_cplx *)a)->im, y = ((const vo_cplx *)b)->im;
    return (x > y) - (x < y);
}

/* Chebyshev-I low-pass as second-order sections, restating
 * designChebyshevI_LP (src/util/downsampling_filter_iir.cpp:58-193) and
 * distributeDCGain (:11-56): bilinear prewarping, order from the ripple /
 * attenuation specs, the N analogue poles sorted by imaginary part and
 * taken two at a time (each pair's first pole with its conjugate gives a
 * section with zeros at z = -1; a last unpaired pole a first-order section),
 * then the DC gain spread over the sections in long double.  sos out
 * [max][6] {b0, b1, b2, a0, a1, a2}; returns the section count, -1 for
 * invalid specs, -2 when max is too small. */
VO_API int vo_cheby_design(double fs, double fc, double fstop, double ap_db, double as_db, double *sos, int max)
{
    if (fs <= 0 || fc <= 0 || fc >= 0.5 * fs) return -1;
    if (fstop <= 0.0) fstop = fmin(0.499 * fs, 1.15 * fc);
    if (fstop <= fc) return -1;
    const double T = 1.0 / fs;
    const double wp = 2.0 / T * tan(M_PI * (fc / fs));
    const double ws = 2.0 / T * tan(M_PI * (fstop / fs));
    const double W = 2.0 / T;
    const double ep = sqrt(pow(10.0, ap_db / 10.0) - 1.0);
    const double x = sqrt((pow(10.0, as_db / 10.0) - 1.0) / (pow(10.0, ap_db / 10.0) - 1.0));
    const double num = log(x + sqrt(x * x - 1.0));                 /* acosh */
    const double r = ws / wp;
    const double den = log(r + sqrt(r * r - 1.0));
    int N = (int)ceil(num / den);
    if (N < 1) N = 1;
    const double ie = 1.0 / ep;
    const double a = log(ie + sqrt(ie * ie + 1.0)) / N;            /* asinh */
    vo_cplx *p = malloc(sizeof(vo_cplx) * (size_t)N);
    if (!p) return -1;
    for (int k = 1; k <= N; ++k) {
        const double theta = M_PI * (2.0 * k - 1.0) / (2.0 * N);
        const double sigma = -sinh(a) * sin(theta);
        const double omega = cosh(a) * cos(theta);
        vo_cplx s = {sigma * wp, omega * wp};
        if (s.re >= 0) s.re = -fabs(s.re);
        p[k - 1] = s;
    }
    qsort(p, (size_t)N, sizeof(vo_cplx), vo_cmp_imag);   /* the imaginary parts are distinct */
    int n = 0;
    for (int i = 0; i < N;) {
        if (n >= max) { free(p); return -2; }
        double *s = sos + 6 * n;
        const vo_cplx q = p[i];
        if (i + 1 == N || fabs(q.im) < 1e-12) {
            const double a0 = W - q.re, a1 = -(W + q.re);
            const double inva0 = 1.0 / a0;
            s[0] = 1.0 * inva0; s[1] = 1.0 * inva0; s[2] = 0.0 * inva0;
            s[3] = 1.0; s[4] = a1 * inva0; s[5] = 0.0 * inva0;
            ++i;
        } else {
            const double are = q.re;
            const double b2 = q.re * q.re + q.im * q.im;         /* |p|^2 */
            const double A0 = (W * W - 2.0 * are * W + b2);
            const double A1 = 2.0 * (b2 - W * W);
            const double A2 = (W * W + 2.0 * are * W + b2);
            const double inva0 = 1.0 / A0;
            s[0] = 1.0 * inva0; s[1] = 2.0 * inva0; s[2] = 1.0 * inva0;
            s[3] = 1.0; s[4] = A1 * inva0; s[5] = A2 * inva0;
            i += 2;
        }
        ++n;
    }
    free(p);
    /* DC gain 1, spread evenly, rounding error folded into section 0 */
    long double H1 = 1.0L;
    for (int i = 0; i < n; ++i) {
        const double *s = sos + 6 * i;
        const long double nu = (long double)s[0] + s[1] + s[2], de = (long double)s[3] + s[4] + s[5];
        H1 *= nu / de;
    }
    if (!isfinite((double)H1) || fabsl(H1) < 1e-300L) return n;
    const long double G = 1.0L / H1;
    const long double g = powl(G, 1.0L / (long double)n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < 3; ++j) sos[6 * i + j] = (double)((long double)sos[6 * i + j] * g);
    long double H1b = 1.0L;
    for (int i = 0; i < n; ++i) {
        const double *s = sos + 6 * i;
        const long double nu = (long double)s[0] + s[1] + s[2], de = (long double)s[3] + s[4] + s[5];
        H1b *= nu / de;
    }
    const long double c = 1.0L / H1b;
    for (int j = 0; j < 3; ++j) sos[j] = (double)((long double)sos[j] * c);
    return n;
}

/* One channel through the cascade from a zero state in FP64, transposed
 * direct form II (processBlock, downsampling_filter_iir.cpp:210-240). */
VO_API void vo_sos_df2t(const double *sos, int n, const float *in, float *out, uint64_t frames)
{
    double z[64][2] = {{0}};
    for (uint64_t t = 0; t < frames; ++t) {
        double y = (double)in[t];
        for (int s = 0; s < n && s < 64; ++s) {
            const double *b = sos + 6 * s;
            const double x = y;
            const double yo = b[0] * x + z[s][0];
            const double z1 = b[1] * x - b[4] * yo + z[s][1];
            const double z2 = b[2] * x - b[5] * yo;
            z[s][0] = z1;
            z[s][1] = z2;
            y = yo;
        }
        out[t] = (float)y;
    }
}

/* Output length for `steps` samples at step dt resampled to `rate`
 * (simulator.cpp:1037-1038). */
VO_API uint64_t vo_resample_len(double rate, uint64_t steps, float dt)
{
    return (uint64_t)(rate * ((double)steps * (double)dt));
}

/* Resampling of one filtered channel by linear interpolation at k / rate
 * (the arithmetic of the interpolation at simulator.cpp:1046-1057: float
 * time, index in double then float), the last sample held past the end;
 * then, if normalize, division by the peak magnitude (simulator.cpp:
 * 1067-1076; a silent channel stays zero).  FP32 with flush-to-zero, as on
 * the GPU. */
VO_API void vo_resample(const float *in, uint64_t len, double sim_rate, double rate, float *out, uint64_t out_len,
                        int normalize)
{
    ftz_on();
    for (uint64_t k = 0; k < out_len; ++k) {
        const float t = (float)k / (float)rate;
        const float index = (float)((double)t * sim_rate);
        uint64_t lo = (uint64_t)floorf(index);
        if (lo >= len) lo = len ? len - 1 : 0;
        const uint64_t hi = lo + 1 < len ? lo + 1 : lo;
        const float frac = index - (float)lo;
        const float a = len ? in[lo] : 0.f, b = len ? in[hi] : 0.f;
        out[k] = a * (1.f - frac) + b * frac;
    }
    if (normalize) {
        float peak = 0.f;
        for (uint64_t k = 0; k < out_len; ++k) peak = fmaxf(peak, fabsf(out[k]));
        if (peak > 0.f)
            for (uint64_t k = 0; k < out_len; ++k) out[k] = out[k] / peak;
    }
    ftz_off();
}

/* An audio signal at `rate` read at step * dt by linear interpolation: the
 * design commented at simulator_gpu.cu:219-231 (float time and index, 0
 * once index + 1 reaches the end of the signal).  IEEE single, no
 * contraction. */
/* The library's band-limited resampler (virs_postprocess_ir_sinc; no
 * reference counterpart: the reference resamples with kfr, absent here):
 * output sample k at input position t = k fs_in / rate is
 * sum_n x[n] 2 fc sinc(2 fc (t - n)) w(t - n) over |t - n| < half, with
 * fc = cutoff min(fs_in, rate) / 2 / fs_in, sinc(u) = sin(pi u) / (pi u) and
 * the Kaiser window w(tau) = I0(beta sqrt(1 - (tau / half)^2)) / I0(beta), I0
 * from its power series; FP64; then division by the peak if asked. */
static double vo_bessel_i0(double x)
{
    const double q = 0.25 * x * x;
    double t = 1.0, s = 1.0;
    for (int k = 1; k < 500; ++k) {
        t = t * q / ((double)k * (double)k);
        s = s + t;
        if (t < 1e-17 * s) break;
    }
    return s;
}

VO_API void vo_resample_sinc(const float *in, uint64_t len, double fs_in, double rate, int half, double beta,
                             double cutoff, float *out, uint64_t out_len, int normalize)
{
    const double fc2 = cutoff * fmin(fs_in, rate) / fs_in, i0b = vo_bessel_i0(beta), ratio = fs_in / rate;
#pragma omp parallel for schedule(static) num_threads(vo_get_threads())
    for (int64_t k = 0; k < (int64_t)out_len; ++k) {
        const double t = (double)k * ratio;
        const double n0 = fmax(0.0, ceil(t - (double)half)), n1 = fmin((double)len - 1.0, floor(t + (double)half));
        double acc = 0.0;
        for (double n = n0; n <= n1; n += 1.0) {
            const double tau = t - n, u = tau / (double)half;
            if (!(fabs(u) < 1.0)) continue;
            const double w = vo_bessel_i0(beta * sqrt(1.0 - u * u)) / i0b;
            const double x = fc2 * tau;
            const double sc = x == 0.0 ? 1.0 : sin(M_PI * x) / (M_PI * x);
            acc += (double)in[(uint64_t)n] * (fc2 * sc * w);
        }
        out[k] = (float)acc;
    }
    if (normalize) {
        float peak = 0.f;
        for (uint64_t k = 0; k < out_len; ++k) peak = fmaxf(peak, fabsf(out[k]));
        if (peak > 0.f)
            for (uint64_t k = 0; k < out_len; ++k) out[k] = out[k] / peak;
    }
}

VO_API void vo_audio_to_steps(const float *x, uint64_t len, float rate, float dt, uint64_t steps, float *out)
{
    for (uint64_t n = 0; n < steps; ++n) {
        const float t = (float)n * dt;
        const float si = t * rate;
        float v = 0.f;
        if (si + 1.f < (float)len) {
            const uint64_t lo = (uint64_t)si;
            const float fr = si - (float)lo;
            v = x[lo] + fr * (x[lo + 1] - x[lo]);
        }
        out[n] = v;
    }
}
