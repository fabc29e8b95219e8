// Voxel classification on the GPU: the sponge-layer distance build, the
// normals bitmask, the cell codes of the step kernel and the compacted,
// ascending boundary-voxel list.
//
// Reference semantics (src/simulator/sponge_kernel.cu:8-62, generalised to
// width W): an interior air voxel (flag 0) becomes a boundary voxel (flag 2)
// when some wall voxel (flag 1) lies in the cube [-W, W]^3 around it with
// squared distance d2 < W*W + 1.  The reference scans the whole cube per
// voxel, (2W+1)^3 flag reads.  Here the minimum is taken one axis at a time
// (three passes of 2W+1 reads each), which is exact because the squared
// distance separates, min over the cube of dx^2+dy^2+dz^2 equals
// min_dz(dz^2 + min_dy(dy^2 + min_dx dx^2)).  Each candidate is carried as
// one packed key
//     d2 << 18 | (dz+32) << 12 | (dy+32) << 6 | (dx+32)
// so that an unsigned minimum picks the smallest d2 and, among equals, the
// first voxel in the reference's scan order (dz, then dy, then dx
// ascending); the offsets of the winner locate the nearest wall voxel, whose
// material becomes the boundary voxel's material.  W <= 31.
#include <algorithm>

#include "internal.hpp"

namespace virs {
namespace {

constexpr uint32_t KINF = 0xffffffffu;

__device__ __forceinline__ bool inside(int x, int y, int z, int nx, int ny, int nz)
{
    return x > 0 && y > 0 && z > 0 && x < nx - 1 && y < ny - 1 && z < nz - 1;
}

// pass 1: along x, from the flags
__global__ void k_edt_x(const uint8_t *__restrict flags, uint32_t *__restrict k1, int nx, int ny, int nz, int px, int W)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    const size_t row = ((size_t)z * ny + y) * px;
    uint32_t best = KINF;
    for (int dx = -W; dx <= W; ++dx) {
        const int xx = x + dx;
        if (xx < 0 || xx >= nx) continue;
        if (__ldg(flags + row + xx) != 1) continue;
        const uint32_t key = ((uint32_t)(dx * dx) << 18) | (uint32_t)(dx + 32);
        best = min(best, key);
    }
    k1[row + x] = best;
}

// pass 2: along y
__global__ void k_edt_y(const uint32_t *__restrict k1, uint32_t *__restrict k2, int nx, int ny, int nz, int px, int W)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    const uint32_t lim = (uint32_t)(W * W);
    uint32_t best = KINF;
    for (int dy = -W; dy <= W; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= ny) continue;
        const uint32_t v = __ldg(k1 + ((size_t)z * ny + yy) * px + x);
        if (v == KINF) continue;
        const uint32_t d2 = (v >> 18) + (uint32_t)(dy * dy);
        if (d2 > lim) continue;
        const uint32_t key = (d2 << 18) | ((uint32_t)(dy + 32) << 6) | (v & 0x3fu);
        best = min(best, key);
    }
    k2[((size_t)z * ny + y) * px + x] = best;
}

// pass 3: along z, then the classification itself
__global__ void k_edt_z(const ClassifyArgs a)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz, px = a.px, W = a.W;
    if (x >= nx) return;
    const size_t i = ((size_t)z * ny + y) * px + x;
    const uint8_t f = a.flags_in[i];
    a.bmat_full[i] = 0;
    a.bd2_full[i] = 0;
    if (f != 0 || !inside(x, y, z, nx, ny, nz)) {
        a.flags_out[i] = f;
        return;
    }
    const uint32_t lim = (uint32_t)(W * W);
    uint32_t best = KINF;
    for (int dz = -W; dz <= W; ++dz) {
        const int zz = z + dz;
        if (zz < 0 || zz >= nz) continue;
        const uint32_t v = __ldg(a.k2 + ((size_t)zz * ny + y) * px + x);
        if (v == KINF) continue;
        const uint32_t d2 = (v >> 18) + (uint32_t)(dz * dz);
        if (d2 > lim) continue;
        const uint32_t key = (d2 << 18) | ((uint32_t)(dz + 32) << 12) | (v & 0xfffu);
        best = min(best, key);
    }
    if (best == KINF) {
        a.flags_out[i] = 0;
        return;
    }
    const int dx = (int)(best & 0x3fu) - 32;
    const int dy = (int)((best >> 6) & 0x3fu) - 32;
    const int dz = (int)((best >> 12) & 0x3fu) - 32;
    const size_t w = ((size_t)(z + dz) * ny + (y + dy)) * px + (x + dx);
    a.flags_out[i] = 2;
    a.bmat_full[i] = a.wall_mat[w];
    a.bd2_full[i] = (uint16_t)(best >> 18);
}

// cell code, normals, per-segment boundary counts and whether a segment
// holds any non-zero code; one block of SEG threads per 128-voxel row
// segment
__global__ void k_codes(const CodesArgs a)
{
    const int x = blockIdx.x * SEG + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz, px = a.px;
    bool bnd = false, nonzero = false;
    if (x < px) {
        const size_t sy = px, sz = (size_t)px * ny;
        const size_t i = (size_t)z * sz + (size_t)y * sy + x;
        uint8_t code = CODE_NONE, nrm = 0;
        if (inside(x, y, z, nx, ny, nz)) {
            const uint8_t *F = a.flags;
            const uint8_t f = F[i];
            // simulator.cpp:480-531
            if (F[i + 1] == 0) nrm |= 1;
            if (F[i - 1] == 0) nrm |= 2;
            if (F[i + sy] == 0) nrm |= 4;
            if (F[i - sy] == 0) nrm |= 8;
            if (F[i + sz] == 0) nrm |= 16;
            if (F[i - sz] == 0) nrm |= 32;
            if (f == 1) code = CODE_WALL;
            else if (f == 3) code = CODE_HARD;
            else if (f == 0 || f == 2) {
                uint8_t m = 0;
                if (F[i + 1] == 1) m |= W_XP;
                if (F[i - 1] == 1) m |= W_XM;
                if (F[i + sy] == 1) m |= W_YP;
                if (F[i - sy] == 1) m |= W_YM;
                if (F[i + sz] == 1) m |= W_ZP;
                if (F[i - sz] == 1) m |= W_ZM;
                code = m | (f == 2 ? CODE_BND : 0);
                bnd = f == 2;
            }
        }
        a.code[i] = code;
        a.normals[i] = nrm;
        nonzero = code != 0;
    }
    const int cnt = __syncthreads_count(bnd);
    const int any = __syncthreads_or(nonzero);
    if (threadIdx.x == 0) {
        a.segcnt[((size_t)z * ny + y) * a.spr + blockIdx.x] = (uint32_t)cnt;
        a.segnz[((size_t)z * ny + y) * a.spr + blockIdx.x] = any ? 1 : 0;
    }
}

// boundary voxels of one segment get consecutive slots after bseg[segment]
__global__ void k_compact(const CompactArgs a)
{
    __shared__ int wsum[SEG / 32];
    const int x = blockIdx.x * SEG + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz, px = a.px;
    const size_t i = ((size_t)z * ny + y) * px + x;
    const bool bnd = x < px && inside(x, y, z, nx, ny, nz) && a.flags[i] == 2;
    const unsigned bal = __ballot_sync(0xffffffffu, bnd);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    if (!bnd) return;
    int before = __popc(bal & ((1u << lane) - 1u));
    for (int w = 0; w < wid; ++w) before += wsum[w];
    const uint64_t slot = (uint64_t)a.bseg[((size_t)z * ny + y) * a.spr + blockIdx.x] + before;
    a.bidx[slot] = (uint32_t)(((uint64_t)z * ny + y) * nx + x);
    a.bpos[slot] = (uint32_t)i;
    a.bcode[slot] = a.code[i];
    a.bnrm[slot] = a.normals[i];
    a.bmat[slot] = a.bmat_full[i];
    a.bw[slot] = a.wtab[a.bd2_full[i]];
}

// ---- exclusive scan (three phases) -------------------------------------------

constexpr int SCAN_B = 1024;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t ws[SCAN_B / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) ws[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < SCAN_B / 32 ? ws[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < SCAN_B / 32) ws[lane] = wi - w;
        if (lane == SCAN_B / 32 - 1) *total = wi;
    }
    __syncthreads();
    return inc - v + ws[wid];
}

__global__ void k_scan_blocks(uint32_t *data, size_t n, uint32_t *bsum)
{
    __shared__ uint32_t tot;
    const size_t i = (size_t)blockIdx.x * SCAN_B + threadIdx.x;
    const uint32_t v = i < n ? data[i] : 0;
    const uint32_t e = block_excl_scan(v, &tot);
    if (i < n) data[i] = e;
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_scan_add(uint32_t *data, size_t n, const uint32_t *boff)
{
    const size_t i = (size_t)blockIdx.x * SCAN_B + threadIdx.x;
    if (i < n) data[i] += boff[blockIdx.x];
}

__global__ void k_scan_total(const uint32_t *data, const uint32_t *orig_last, size_t n, uint32_t *total)
{
    *total = data[n - 1] + *orig_last;
}

__global__ void k_copy1(const uint32_t *src, uint32_t *dst) { *dst = *src; }

} // namespace

cudaError_t launch_sponge(const ClassifyArgs &a, cudaStream_t s)
{
    const dim3 blk(128);
    const dim3 grd((a.nx + 127) / 128, a.ny, a.nz);
    k_edt_x<<<grd, blk, 0, s>>>(a.flags_in, a.k1, a.nx, a.ny, a.nz, a.px, a.W);
    k_edt_y<<<grd, blk, 0, s>>>(a.k1, a.k2, a.nx, a.ny, a.nz, a.px, a.W);
    k_edt_z<<<grd, blk, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_codes(const CodesArgs &a, cudaStream_t s)
{
    k_codes<<<dim3(a.spr, a.ny, a.nz), dim3(SEG), 0, s>>>(a);
    return cudaGetLastError();
}

size_t scan_tmp_words(size_t n)
{
    size_t words = 1;
    do {
        n = (n + SCAN_B - 1) / SCAN_B;
        words += n;
    } while (n > 1);
    return words;
}

namespace {
// exclusive scan of data[0..n) in place; tmp holds the per-block sums of
// every level
cudaError_t scan_levels(uint32_t *data, size_t n, uint32_t *tmp, cudaStream_t s)
{
    const size_t nb = (n + SCAN_B - 1) / SCAN_B;
    uint32_t *bsum = tmp;
    k_scan_blocks<<<(unsigned)nb, SCAN_B, 0, s>>>(data, n, bsum);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || nb == 1) return e;
    e = scan_levels(bsum, nb, tmp + nb, s);
    if (e != cudaSuccess) return e;
    k_scan_add<<<(unsigned)nb, SCAN_B, 0, s>>>(data, n, bsum);
    return cudaGetLastError();
}
} // namespace

// data[0..n) <- exclusive prefix sums; *total <- their sum.
cudaError_t launch_scan(uint32_t *data, size_t n, uint32_t *tmp, uint32_t *total, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_copy1<<<1, 1, 0, s>>>(data + n - 1, tmp); // the last input, for the total
    cudaError_t e = scan_levels(data, n, tmp + 1, s);
    if (e != cudaSuccess) return e;
    k_scan_total<<<1, 1, 0, s>>>(data, tmp, n, total);
    return cudaGetLastError();
}

namespace {
// device positions of the hard-source voxels (code CODE_HARD); with
// out == nullptr only counts them.  The order is arbitrary: every step
// writes the same value to all of them.
__global__ void k_hard_list(const uint8_t *__restrict code, uint64_t n, uint32_t *count, uint32_t *out, uint32_t cap)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (code[i] == CODE_HARD) {
            const uint32_t k = atomicAdd(count, 1u);
            if (out && k < cap) out[k] = (uint32_t)i;
        }
}
} // namespace

cudaError_t launch_hard_list(const uint8_t *code, uint64_t n, uint32_t *count, uint32_t *out, uint32_t cap,
                             cudaStream_t s)
{
    k_hard_list<<<1184, 256, 0, s>>>(code, n, count, out, cap);
    return cudaGetLastError();
}

cudaError_t launch_compact(const CompactArgs &a, cudaStream_t s)
{
    k_compact<<<dim3(a.spr, a.ny, a.nz), dim3(SEG), 0, s>>>(a);
    return cudaGetLastError();
}


// ---- planes of a stencil tile whose codes are all zero ---------------------------
//
// For a rows x zc tiling, bit j of a tile's mask is set when the codes of
// the plane staged in stage j (plane z0 - 1 + j, j < 64, one of the tile's
// own planes) are all zero over the tile's 128 x rows voxels: the stencil
// then skips their copy and treats every voxel as plain air.  From the
// per-segment flags of k_codes (a tile row is one segment).
namespace {
__global__ void __launch_bounds__(64) k_tile_zero_mask(const uint8_t *__restrict segnz, uint32_t ny, uint32_t nz,
                                                       uint32_t spr, uint32_t rows, uint32_t zc, uint32_t gx,
                                                       uint32_t gy, uint32_t zb, uint32_t ze,
                                                       uint64_t *__restrict mask)
{
    __shared__ unsigned w[2];
    const uint32_t t = blockIdx.x, j = threadIdx.x;
    const uint32_t bx = t % gx, by = (t / gx) % gy, bz = t / (gx * gy);
    const uint32_t z0 = zb + bz * zc, z1 = min(z0 + zc, ze);
    const uint32_t k = z0 - 1 + j;
    bool zero = false;
    if (k >= z0 && k < z1) {
        zero = true;
        const uint32_t y1 = min(by * rows + rows, ny);
        for (uint32_t y = by * rows; y < y1 && zero; ++y) zero = segnz[((size_t)k * ny + y) * spr + bx] == 0;
    }
    const unsigned b = __ballot_sync(0xffffffffu, zero);
    if ((j & 31) == 0) w[j >> 5] = b;
    __syncthreads();
    if (j == 0) mask[t] = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
}
} // namespace

cudaError_t launch_tile_zero_masks(const uint8_t *segnz, uint32_t ny, uint32_t nz, uint32_t spr, uint32_t rows,
                                   uint32_t zc, uint32_t gx, uint32_t gy, uint32_t gz, uint32_t zb, uint32_t ze,
                                   uint64_t *mask, cudaStream_t s)
{
    const uint64_t ntiles = (uint64_t)gx * gy * gz;
    if (ntiles == 0) return cudaSuccess;
    k_tile_zero_mask<<<(unsigned)ntiles, 64, 0, s>>>(segnz, ny, nz, spr, rows, zc, gx, gy, zb, ze, mask);
    return cudaGetLastError();
}

// The same masks for the tiles of the two-step kernel: a tile covers x in
// [bx*ix - v, bx*ix - v + 128) and rows [by*iy - 1, by*iy - 1 + rows) (the
// parts outside the grid read as code 0), and stage j holds plane
// zs - 2 + j with zs = 1 + bz*zc; the stages with codes are the planes
// zs-1 .. z1.  A bit is set when every 128-voxel segment the tile's codes
// touch on that plane holds only zeros.
namespace {
__global__ void __launch_bounds__(64) k_pair_zero_mask(const uint8_t *__restrict segnz, uint32_t px, uint32_t ny,
                                                       uint32_t nz, uint32_t spr, uint32_t rows, uint32_t zc,
                                                       uint32_t ix, uint32_t v, uint32_t gx, uint32_t gy,
                                                       uint64_t *__restrict mask)
{
    __shared__ unsigned w[2];
    const uint32_t t = blockIdx.x, j = threadIdx.x;
    const uint32_t bx = t % gx, by = (t / gx) % gy, bz = t / (gx * gy);
    const int zs = 1 + (int)(bz * zc), z1 = min(zs + (int)zc, (int)nz - 1);
    const int k = zs - 2 + (int)j;
    bool zero = false;
    if (k >= zs - 1 && k <= z1 && k >= 0 && k < (int)nz) {
        zero = true;
        const int xs = (int)(bx * ix) - (int)v, ys = (int)(by * (rows - 2)) - 1;
        const int xa = max(xs, 0), xb = min(xs + 128, (int)px);
        const int ya = max(ys, 0), yb = min(ys + (int)rows, (int)ny);
        for (int y = ya; y < yb && zero; ++y)
            for (int sx = xa / 128; sx <= (xb - 1) / 128 && zero; ++sx)
                zero = segnz[((size_t)k * ny + y) * spr + sx] == 0;
    }
    const unsigned b = __ballot_sync(0xffffffffu, zero);
    if ((j & 31) == 0) w[j >> 5] = b;
    __syncthreads();
    if (j == 0) mask[t] = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
}
} // namespace

cudaError_t launch_pair_zero_masks(const uint8_t *segnz, uint32_t px, uint32_t ny, uint32_t nz, uint32_t spr,
                                   uint32_t rows, uint32_t zc, uint32_t ix, uint32_t v, uint32_t gx, uint32_t gy,
                                   uint32_t gz, uint64_t *mask, cudaStream_t s)
{
    const uint64_t ntiles = (uint64_t)gx * gy * gz;
    if (ntiles == 0) return cudaSuccess;
    k_pair_zero_mask<<<(unsigned)ntiles, 64, 0, s>>>(segnz, px, ny, nz, spr, rows, zc, ix, v, gx, gy, mask);
    return cudaGetLastError();
}

// ---- voxels whose second step of a two-step pass is provisional --------------
//
// The two-step stencil computes p^{n+2} from p^{n+1} before the boundary
// pass and the post kernel have changed p^{n+1} at boundary voxels and
// sources.  The p^{n+2} of every voxel the stencil updates (air or mirror
// code: bit 7 clear) that is such a voxel or its face neighbour must be
// recomputed afterwards.  k_pair_mark marks them, k_mark_count counts the
// marks of each 1024-voxel segment, and after an exclusive scan of the
// counts k_mark_list writes their positions in ascending order.
namespace {
constexpr int MARK_B = 1024;

__device__ __forceinline__ void mark_around(const uint8_t *__restrict code, uint8_t *mark, uint64_t v, uint32_t px,
                                            uint32_t ny, uint32_t nz)
{
    const uint64_t plane = (uint64_t)px * ny;
    const uint32_t x = (uint32_t)(v % px), y = (uint32_t)((v / px) % ny), z = (uint32_t)(v / plane);
    if (z >= nz) return;
    const uint64_t nbv[7] = {v, v + 1, v - 1, v + px, v - px, v + plane, v - plane};
    const bool in[7] = {true, x + 1 < px, x > 0, y + 1 < ny, y > 0, z + 1 < nz, z > 0};
#pragma unroll
    for (int k = 0; k < 7; ++k)
        if (in[k] && (code[nbv[k]] & CODE_BND) == 0) mark[nbv[k]] = 1;
}

__global__ void k_pair_mark(const uint8_t *__restrict code, uint32_t px, uint32_t ny, uint32_t nz,
                            const uint32_t *__restrict bpos, uint64_t nb, const uint32_t *__restrict hpos, uint32_t nh,
                            const uint64_t *__restrict src, uint32_t nsrc, uint8_t *mark)
{
    const uint64_t n = nb + nh + nsrc;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = i < nb ? (uint64_t)bpos[i] : i < nb + nh ? (uint64_t)hpos[i - nb] : src[i - nb - nh];
        mark_around(code, mark, v, px, ny, nz);
    }
}

__global__ void __launch_bounds__(MARK_B) k_mark_count(const uint8_t *__restrict mark, uint64_t n, uint32_t *cnt)
{
    const uint64_t i = (uint64_t)blockIdx.x * MARK_B + threadIdx.x;
    const int c = __syncthreads_count(i < n && mark[i] != 0);
    if (threadIdx.x == 0) cnt[blockIdx.x] = (uint32_t)c;
}

__global__ void __launch_bounds__(MARK_B) k_mark_list(const uint8_t *__restrict mark, uint64_t n,
                                                      const uint32_t *__restrict off, uint32_t *list)
{
    __shared__ uint32_t tot;
    const uint64_t i = (uint64_t)blockIdx.x * MARK_B + threadIdx.x;
    const uint32_t f = i < n && mark[i] != 0 ? 1u : 0u;
    const uint32_t e = block_excl_scan(f, &tot);
    if (f) list[off[blockIdx.x] + e] = (uint32_t)i;
}
} // namespace

size_t mark_segments(uint64_t nvox) { return (size_t)((nvox + MARK_B - 1) / MARK_B); }

cudaError_t launch_pair_marks(const uint8_t *code, uint32_t px, uint32_t ny, uint32_t nz, const uint32_t *bpos,
                              uint64_t nb, const uint32_t *hpos, uint32_t nh, const uint64_t *src, uint32_t nsrc,
                              uint8_t *mark, uint32_t *cnt, cudaStream_t s)
{
    const uint64_t nvox = (uint64_t)px * ny * nz;
    if (nb + nh + nsrc) {
        const uint64_t n = nb + nh + nsrc;
        const unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
        k_pair_mark<<<g, 256, 0, s>>>(code, px, ny, nz, bpos, nb, hpos, nh, src, nsrc, mark);
    }
    k_mark_count<<<(unsigned)mark_segments(nvox), MARK_B, 0, s>>>(mark, nvox, cnt);
    return cudaGetLastError();
}

cudaError_t launch_mark_list(const uint8_t *mark, uint64_t nvox, const uint32_t *off, uint32_t *list, cudaStream_t s)
{
    k_mark_list<<<(unsigned)mark_segments(nvox), MARK_B, 0, s>>>(mark, nvox, off, list);
    return cudaGetLastError();
}

} // namespace virs
