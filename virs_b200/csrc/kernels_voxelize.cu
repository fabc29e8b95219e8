// Mesh -> voxel flags on the GPU (the reference sweeps the triangles on the
// host, simulator.cpp:396-452).
//
//   k_tri_prep    per triangle: vertices in voxel units (toVoxel,
//                 simulator.h:39-45), the clamped integer bounding box and
//                 the role of its material
//   k_tri_sweep   every (triangle, voxel of its box) pair: the
//                 triangle/box separating-axis test (simulator.cpp:45-141);
//                 a hit raises the voxel's "last triangle" marks with an
//                 atomic maximum of the triangle number
//   k_resolve     marks -> flags and wall materials
// The grid may be a window of planes [zw, zw + nzl) of a taller grid (a
// z-slab): voxel coordinates and the cell tests stay global, so every hit
// is the whole grid's, and only the boxes and the stored index are cut to
// the window.
// The reference's sweep runs the triangles in order and a later triangle
// overwrites a voxel's flag (wall 1 or source 3), while a source triangle
// leaves the wall material alone.  So the flag comes from the last wall or
// source triangle that hits the voxel and the wall material from the last
// wall triangle: two maxima per voxel give exactly that, in any order of
// execution.
//
// This file is compiled with -fmad=false and without flush-to-zero: every
// float expression is evaluated as written in IEEE single precision, as on
// the host (-ffp-contract=off), so the hits are the host's bit for bit.
#include "internal.hpp"

namespace virs {
namespace {

struct Tri {
    float g[9];   // vertices in voxel units
    int box[6];   // ix0, iy0, iz0, ix1, iy1, iz1 (inclusive)
    uint32_t role;
};

struct F3 {
    float x, y, z;
};

__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 abs3(F3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
__device__ __forceinline__ float mn3(float a, float b, float c)
{
    float m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    return m;
}
__device__ __forceinline__ float mx3(float a, float b, float c)
{
    float m = a;
    if (m < b) m = b;
    if (m < c) m = c;
    return m;
}

// one edge/axis test; the projection uses the .y and .z components for every
// pair, as the reference's test does (simulator.cpp:73-86)
__device__ __forceinline__ bool axis(float a, float b, float fa, float fb, F3 p0, F3 p1, F3 p2, float ex, float ey)
{
    const float q0 = a * p0.y - b * p0.z, q1 = a * p1.y - b * p1.z, q2 = a * p2.y - b * p2.z;
    const float lo = mn3(q0, q1, q2), hi = mx3(q0, q1, q2);
    const float rad = fa * ey + fb * ex;
    return !(lo > rad || hi < -rad);
}

// triangle (voxel units) against the unit cell [i, i+1] x [j, j+1] x [k, k+1]
__device__ bool overlap(const float *g, float i, float j, float k)
{
    const F3 lo = {i, j, k}, hi = {i + 1.f, j + 1.f, k + 1.f};
    const F3 c = {(lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f};
    const F3 e = {(hi.x - lo.x) * 0.5f, (hi.y - lo.y) * 0.5f, (hi.z - lo.z) * 0.5f};
    const F3 v0 = sub3({g[0], g[1], g[2]}, c), v1 = sub3({g[3], g[4], g[5]}, c), v2 = sub3({g[6], g[7], g[8]}, c);
    const F3 f0 = sub3(v1, v0), f1 = sub3(v2, v1), f2 = sub3(v0, v2);
    const F3 a0 = abs3(f0), a1 = abs3(f1), a2 = abs3(f2);
    if (!axis(f0.z, f0.y, a0.z, a0.y, v0, v1, v2, e.y, e.z)) return false;
    if (!axis(f0.z, f0.x, a0.z, a0.x, v0, v1, v2, e.x, e.z)) return false;
    if (!axis(f0.y, f0.x, a0.y, a0.x, v0, v1, v2, e.x, e.y)) return false;
    if (!axis(f1.z, f1.y, a1.z, a1.y, v0, v1, v2, e.y, e.z)) return false;
    if (!axis(f1.z, f1.x, a1.z, a1.x, v0, v1, v2, e.x, e.z)) return false;
    if (!axis(f1.y, f1.x, a1.y, a1.x, v0, v1, v2, e.x, e.y)) return false;
    if (!axis(f2.z, f2.y, a2.z, a2.y, v0, v1, v2, e.y, e.z)) return false;
    if (!axis(f2.z, f2.x, a2.z, a2.x, v0, v1, v2, e.x, e.z)) return false;
    if (!axis(f2.y, f2.x, a2.y, a2.x, v0, v1, v2, e.x, e.y)) return false;
    float m = mn3(v0.x, v1.x, v2.x), M = mx3(v0.x, v1.x, v2.x);
    if (m > e.x || M < -e.x) return false;
    m = mn3(v0.y, v1.y, v2.y);
    M = mx3(v0.y, v1.y, v2.y);
    if (m > e.y || M < -e.y) return false;
    m = mn3(v0.z, v1.z, v2.z);
    M = mx3(v0.z, v1.z, v2.z);
    if (m > e.z || M < -e.z) return false;
    const F3 n = {f0.y * f1.z - f0.z * f1.y, f0.z * f1.x - f0.x * f1.z, f0.x * f1.y - f0.y * f1.x};
    const float d = -(n.x * v0.x + n.y * v0.y + n.z * v0.z);
    const float r = e.x * fabsf(n.x) + e.y * fabsf(n.y) + e.z * fabsf(n.z);
    return !(fabsf(d) > r);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__global__ void k_tri_prep(const float *__restrict verts, const uint32_t *__restrict tris,
                           const int32_t *__restrict tri_mat, uint64_t ntri, const uint8_t *__restrict roles,
                           uint32_t nroles, float h, float bx, float by, float bz, int nx, int ny, int nz, int zw,
                           int nzl, Tri *__restrict out)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntri) return;
    Tri T;
    for (int c = 0; c < 3; ++c) {
        const float *p = verts + 3 * (uint64_t)tris[3 * t + c];
        T.g[3 * c + 0] = (p[0] - bx) / h;
        T.g[3 * c + 1] = (p[1] - by) / h;
        T.g[3 * c + 2] = (p[2] - bz) / h;
    }
    const int mid = tri_mat[t];
    T.role = (mid >= 0 && (uint32_t)mid < nroles) ? roles[mid] : VIRS_ROLE_IGNORE;
    const int n[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        T.box[a] = clampi((int)floorf(mn3(T.g[a], T.g[3 + a], T.g[6 + a])), 0, n[a] - 1);
        T.box[3 + a] = clampi((int)ceilf(mx3(T.g[a], T.g[3 + a], T.g[6 + a])), 0, n[a] - 1);
    }
    // the window of planes held
    T.box[2] = T.box[2] > zw ? T.box[2] : zw;
    T.box[5] = T.box[5] < zw + nzl - 1 ? T.box[5] : zw + nzl - 1;
    if (T.box[2] > T.box[5]) T.role = VIRS_ROLE_IGNORE;
    out[t] = T;
}

// blocks stride over the triangles (x) and over the cells of a triangle's
// box (y and the threads)
__global__ void __launch_bounds__(256) k_tri_sweep(const Tri *__restrict tris, uint64_t ntri, uint32_t px,
                                                   uint32_t ny, int zw, uint32_t *__restrict last_any,
                                                   uint32_t *__restrict last_wall)
{
    for (uint64_t t = blockIdx.x; t < ntri; t += gridDim.x) {
        const Tri &T = tris[t];
        const uint32_t role = T.role;
        if (role == VIRS_ROLE_IGNORE) continue;
        float g[9];
        for (int c = 0; c < 9; ++c) g[c] = T.g[c];
        const int x0 = T.box[0], y0 = T.box[1], z0 = T.box[2];
        const uint64_t sx = (uint64_t)(T.box[3] - x0 + 1), sy = (uint64_t)(T.box[4] - y0 + 1);
        const uint64_t total = sx * sy * (uint64_t)(T.box[5] - z0 + 1);
        for (uint64_t q = (uint64_t)blockIdx.y * blockDim.x + threadIdx.x; q < total;
             q += (uint64_t)gridDim.y * blockDim.x) {
            const int i = x0 + (int)(q % sx), j = y0 + (int)((q / sx) % sy), k = z0 + (int)(q / (sx * sy));
            if (!overlap(g, (float)i, (float)j, (float)k)) continue;
            const size_t idx = ((size_t)(k - zw) * ny + (size_t)j) * px + (size_t)i;
            atomicMax(last_any + idx, (uint32_t)(t + 1));
            if (role != VIRS_ROLE_SOURCE) atomicMax(last_wall + idx, (uint32_t)(t + 1));
        }
    }
}

__global__ void k_resolve(const Tri *__restrict tris, const uint32_t *__restrict last_any,
                          const uint32_t *__restrict last_wall, uint64_t n, uint8_t *__restrict flags,
                          uint8_t *__restrict wall_mat, uint32_t *__restrict max_mat)
{
    uint32_t mx = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = last_any[i], w = last_wall[i];
        if (a) flags[i] = tris[a - 1].role == VIRS_ROLE_SOURCE ? 3 : 1;
        if (w) {
            const uint32_t r = tris[w - 1].role;
            wall_mat[i] = (uint8_t)r;
            mx = r > mx ? r : mx;
        }
    }
    if (mx) atomicMax(max_mat, mx);
}

} // namespace

size_t voxelize_tri_bytes() { return sizeof(Tri); }

cudaError_t launch_voxelize(const float *verts, const uint32_t *tris, const int32_t *tri_mat, uint64_t ntri,
                            const uint8_t *roles, uint32_t nroles, float h, const float bmin[3], uint32_t nx,
                            uint32_t ny, uint32_t nz, uint32_t zw, uint32_t nzl, uint32_t px, void *tri_buf,
                            uint32_t *last_any, uint32_t *last_wall, uint8_t *flags, uint8_t *wall_mat,
                            uint32_t *max_mat, cudaStream_t s)
{
    if (ntri == 0) return cudaSuccess;
    Tri *T = static_cast<Tri *>(tri_buf);
    k_tri_prep<<<(unsigned)((ntri + 127) / 128), 128, 0, s>>>(verts, tris, tri_mat, ntri, roles, nroles, h, bmin[0],
                                                              bmin[1], bmin[2], (int)nx, (int)ny, (int)nz, (int)zw,
                                                              (int)nzl, T);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const unsigned gx = (unsigned)(ntri < 4096 ? ntri : 4096);
    const unsigned gy = ntri < 64 ? 256u : (ntri < 1024 ? 16u : 1u);
    k_tri_sweep<<<dim3(gx, gy), 256, 0, s>>>(T, ntri, px, ny, (int)zw, last_any, last_wall);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const uint64_t n = (uint64_t)px * ny * nzl;
    k_resolve<<<1184, 256, 0, s>>>(T, last_any, last_wall, n, flags, wall_mat, max_mat);
    return cudaGetLastError();
}

} // namespace virs
