// The FDTD step on the GPU: the register-streaming stencil (the variant
// with pipeline depth 0; the TMA-staged default is kernels_step_tma.cu), the
// boundary pass and the per-step source / receiver kernel.
//
// Semantics follow the reference step (src/simulator/simulator_gpu.cu):
//   interior leapfrog with the wall mirror rule       :38-103
//   boundary biquad correction, evaluated in double   :105-150
// in two passes.  Layout and mapping:
//   * fields are [nz][ny][px] with px = nx rounded up to 32 (rows start on
//     128-byte lines); two buffers, p^{n+1} overwrites p^{n-1} in place
//     (each output depends on p^{n-1} at its own voxel only);
//   * a block owns a tile of TX = 32*VEC columns x TY rows and streams it
//     along z over `zc` planes: p at z-1, z, z+1 live in registers, the
//     plane z of the tile (plus one halo row above and below) sits in shared
//     memory for the y neighbours, x neighbours come from warp shuffles and
//     two halo loads per row; every load of plane z+1 is issued one plane
//     ahead of its use;
//   * one byte per voxel (the cell code) replaces the flags and the six
//     neighbour flags of the reference;
//   * boundary voxels (flag 2) are skipped -- their p^{n-1} stays in place --
//     and updated by k_boundary, one thread per entry of the compacted,
//     ascending boundary list: the leapfrog and the biquad correction
//     together, with no divergence in the stencil kernel; the filter states
//     are stored in 16-byte groups per slot (state_index in internal.hpp) so
//     a warp touches consecutive vectors.
//
// Arithmetic order is fixed with _rn intrinsics so that the result is
// bit-identical to the CPU oracle: the reference CUDA build contracts
// s - 6*p and t + c2dt2*lap into fused multiply-adds and flushes subnormals
// (--use_fast_math); this file is compiled with -ftz=true.
#include "step_common.cuh"

namespace virs {
namespace {

using namespace step;

template <typename T, int TY>
__global__ void __launch_bounds__(32 * TY, 1024 / (32 * TY)) k_step(const __grid_constant__ StepArgs a)
{
    using IO = Io<T>;
    constexpr int VEC = IO::VEC;
    constexpr int TX = 32 * VEC;
    __shared__ __align__(16) float sm[2][TY + 2][TX];

    const int lane = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * TX;
    const int x = x0 + lane * VEC;
    const int y0 = blockIdx.y * TY;
    const int y = y0 + ty;
    if (a.stop && *a.stop) return; // the stop rule fired at an earlier step
    const int z0 = a.zb + blockIdx.z * a.zc;
    const int z1 = min(z0 + a.zc, a.ze);
    if (z0 >= z1) return; // uniform over the block

    const int px = (int)a.px, ny = (int)a.ny;
    const bool xin = x < px;
    const bool act = xin && y < ny;
    const size_t plane = (size_t)px * ny;
    const T *P = static_cast<const T *>(a.p);
    T *Q = static_cast<T *>(a.q);
    const size_t own = (size_t)y * px + x;

    // warp 0 also carries the halo row above the tile, the last warp the one below
    int hslot = -1, hrow = 0;
    if (ty == 0 && y0 >= 1) { hslot = 0; hrow = y0 - 1; }
    if (ty == TY - 1 && y0 + TY < ny) { hslot = TY + 1; hrow = y0 + TY; }
    const bool hact = hslot >= 0 && xin;
    const size_t hoff = (size_t)hrow * px + x;
    const bool has_l = lane == 0 && x0 >= 1;
    const bool has_r = lane == 31 && x0 + TX < px;

    for (int i = threadIdx.y * 32 + lane; i < 2 * (TY + 2) * TX; i += 32 * TY) (&sm[0][0][0])[i] = 0.f;
    __syncthreads();

    float cm[VEC], cc[VEC], cp[VEC], qv[VEC], qn[VEC], hv[VEC];
    uint8_t cd[VEC], cdn[VEC];
    float hl = 0.f, hr = 0.f, hln = 0.f, hrn = 0.f;
#pragma unroll
    for (int k = 0; k < VEC; ++k) { cm[k] = cc[k] = cp[k] = qv[k] = qn[k] = hv[k] = 0.f; cd[k] = cdn[k] = CODE_NONE; }

    {
        const size_t zo = (size_t)z0 * plane;
        if (act) {
            IO::ld(P + zo - plane + own, cm);
            IO::ld(P + zo + own, cc);
            IO::ld_stream(Q + zo + own, qv);
            ld_code<VEC>(a.code + zo + own, cd);
            if (has_l) hl = IO::ld1(P + zo + own - 1);
            if (has_r) hr = IO::ld1(P + zo + own + VEC);
#pragma unroll
            for (int k = 0; k < VEC; ++k) sm[0][ty + 1][lane * VEC + k] = cc[k];
        }
        if (hact) {
            IO::ld(P + zo + hoff, hv);
#pragma unroll
            for (int k = 0; k < VEC; ++k) sm[0][hslot][lane * VEC + k] = hv[k];
        }
    }
    __syncthreads();

    const uint32_t srk = a.sr ? sr_step_key(*a.ctr, 0u) : 0u;
    for (int z = z0; z < z1; ++z) {
        const int b = (z - z0) & 1;
        const size_t zc = (size_t)z * plane, zn = zc + plane;
        // loads for plane z+1, consumed in the next iteration
        if (act) {
            IO::ld(P + zn + own, cp);
            if (z + 1 < z1) {
                IO::ld_stream(Q + zn + own, qn);
                ld_code<VEC>(a.code + zn + own, cdn);
            }
            if (has_l) hln = IO::ld1(P + zn + own - 1);
            if (has_r) hrn = IO::ld1(P + zn + own + VEC);
        }
        if (hact) IO::ld(P + zn + hoff, hv);

        float left = __shfl_up_sync(FULL, cc[VEC - 1], 1);
        float right = __shfl_down_sync(FULL, cc[0], 1);
        if (lane == 0) left = hl;
        if (lane == 31) right = hr;

        float r[VEC];
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
            const uint8_t c = cd[k];
            const float ym = sm[b][ty][lane * VEC + k];
            const float yp = sm[b][ty + 2][lane * VEC + k];
            const float xm = k == 0 ? left : cc[k - 1];
            const float xp = k == VEC - 1 ? right : cc[k + 1];
            if (c == CODE_WALL) {
                r[k] = 0.f;
            } else if (c & CODE_BND) {
                r[k] = qv[k]; // border and hard-source voxels keep theirs, the boundary pass updates boundary voxels
            } else {
                r[k] = leapfrog(c, cc[k], xp, xm, yp, ym, cp[k], cm[k], qv[k], a.c2dt2, a.inv_h2);
            }
        }

        if (act) {
            if (a.sr) st_sr<T>(Q + zc + own, r, zc + own, a.sr_base, srk);
            else IO::st(Q + zc + own, r);
#pragma unroll
            for (int k = 0; k < VEC; ++k) sm[b ^ 1][ty + 1][lane * VEC + k] = cp[k];
        }
        if (hact) {
#pragma unroll
            for (int k = 0; k < VEC; ++k) sm[b ^ 1][hslot][lane * VEC + k] = hv[k];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
            cm[k] = cc[k];
            cc[k] = cp[k];
            qv[k] = qn[k];
            cd[k] = cdn[k];
        }
        hl = hln;
        hr = hrn;
    }
}

// The compacted boundary pass (simulator_gpu.cu:105-150): one thread per
// boundary voxel in list order.  The stencil kernels left these voxels
// untouched (p^{n-1} in place); the pass gathers the seven p values and
// p^{n-1} of its voxel, computes the leapfrog update with the wall mirror,
// then the filter correction.  Consecutive slots are consecutive voxels of
// a row (floor, ceiling and y walls) or the same x of consecutive rows
// (x walls), so the gathers of a warp share lines.
//   BND_UPDATE  leapfrog + filters, the result written to p^{n+1}
//   BND_KEEP    the same, and the record {free value, p, p^{n-1}} of the
//               slot kept in a.side (the adjoint's recomputation)
//   BND_RECORD  the record only: no filters, nothing written to the fields
//               (the adjoint step, on adjoint fields)
// The loads of one boundary voxel (first part) and its update (second).
template <typename T, int MAXS> struct BVox {
    size_t i;
    uint8_t c, nm;
    float ce, qv, nb[6];
    BState<MAXS> st;
};

template <typename T, int MODE, int MAXS>
__device__ __forceinline__ void bvox_load(const StepArgs &a, uint64_t slot, BVox<T, MAXS> &v)
{
    using IO = Io<T>;
    const size_t i = __ldg(a.bpos + slot);
    const size_t sy = a.px, sz = (size_t)a.px * a.ny;
    const T *P = static_cast<const T *>(a.p);
    const T *Q = static_cast<const T *>(a.q);
    v.i = i;
    v.c = __ldg(a.bcode + slot);
    v.nm = a.rigid ? __ldg(a.bnrm + slot) : 0;
    v.ce = IO::get(P[i]);
    v.qv = IO::get(Q[i]);
    v.nb[0] = IO::get(P[i + 1]);
    v.nb[1] = IO::get(P[i - 1]);
    v.nb[2] = IO::get(P[i + sy]);
    v.nb[3] = IO::get(P[i - sy]);
    v.nb[4] = IO::get(P[i + sz]);
    v.nb[5] = IO::get(P[i - sz]);
    if (MODE != BND_RECORD && MAXS > 0) bload<MAXS>(a, slot, v.st);
}

template <typename T, int MODE, int MAXS>
__device__ __forceinline__ void bvox_update(const StepArgs &a, uint64_t slot, const BVox<T, MAXS> &v)
{
    float r;
    if (a.rigid) {
        // fdtd_kernel_rigid_walls (simulator_gpu.cu:152-180): the air
        // neighbours only (normals mask), p+ = (2 - l2 n) p - p- + the sum
        // of (l2 * s) * p_nb over +x, -x, +y, -y, +z, -z with s = 1 for air;
        // with the reference build's contractions
        const float b1 = __fmaf_rn(-a.l2, (float)__popc(v.nm), 2.f);
        r = __fmaf_rn(b1, v.ce, -v.qv);
#pragma unroll
        for (int k = 0; k < 6; ++k) r = __fmaf_rn(__fmul_rn(a.l2, (v.nm & (1u << k)) ? 1.f : 0.f), v.nb[k], r);
    } else {
        r = leapfrog(v.c, v.ce, v.nb[0], v.nb[1], v.nb[2], v.nb[3], v.nb[4], v.nb[5], v.qv, a.c2dt2, a.inv_h2);
    }
    if (MODE != BND_UPDATE) a.side[slot] = make_float4(r, v.ce, v.qv, 0.f);
    if (MODE == BND_RECORD) return;
    r = MAXS > 0 ? bcompute<MAXS>(a, r, v.ce, v.qv, slot, v.st) : boundary_loop(a, r, v.ce, v.qv, slot);
    static_cast<T *>(a.q)[v.i] =
        put_rounded<T>(r, a.sr, v.i, a.sr_base, a.sr ? sr_step_key(*a.ctr, 0u) : 0u);
}

// The compacted boundary pass (simulator_gpu.cu:105-150), in list order.
// The stencil kernels left these voxels untouched (p^{n-1} in place); the
// pass gathers the seven p values from the p^n buffer (not written during
// the step) and p^{n-1}, reads the voxel's code from the per-slot copy made
// at classification (in slot order: no 32-byte sector fetched for one
// byte), computes the leapfrog update with the wall mirror (or the
// rigid-wall update), then the filter correction, and writes p^{n+1}.  One
// slot per thread: on the hall, two, three and four slots per thread (all
// loads issued before any arithmetic) measured 3, 8 and 16 % slower, and
// staging the loads of later slots in shared memory slower still.
//   BND_UPDATE  the step
//   BND_KEEP    the same, and the record {free value, p, p^{n-1}} of the
//               slot kept in a.side (the adjoint's recomputation)
//   BND_RECORD  the record only: no filters, nothing written to the fields
//               (the adjoint step, on adjoint fields)
constexpr int BT = 256;

template <typename T, int MODE, int MAXS>
__global__ void __launch_bounds__(BT) k_boundary(const __grid_constant__ StepArgs a)
{
    if (a.stop && *a.stop) return; // the stop rule fired at an earlier step
    const uint64_t s0 = (uint64_t)blockIdx.x * BT + threadIdx.x;
    if (s0 >= a.nb) return;
    BVox<T, MAXS> v;
    bvox_load<T, MODE, MAXS>(a, s0, v);
    bvox_update<T, MODE, MAXS>(a, s0, v);
}

// The second step of a two-step pass (kernels_step_tma.cu, k_pair_tma):
// its boundary pass and the recomputation of its provisional voxels, in one
// launch.  Blocks [0, gb) take boundary slots as k_boundary does; the others
// take entries of the provisional-voxel list: air and mirror voxels at or
// next to a voxel whose p^{n+1} the first step's boundary pass or post
// kernel changed, whose p^{n+2} the two-step kernel computed from the
// provisional p^{n+1}.  They are recomputed from the final p^{n+1} (a.p) and
// p^n (pn) with leapfrog(code, ...), which is bit-identical to the air
// update for code 0 and is the mirror update for the others.  Both parts
// read p^{n+1} and write disjoint voxels of p^{n+2} (a.q): boundary voxels,
// and air or mirror voxels.  One entry per thread, as in the boundary pass.
template <typename T> struct FixVox {
    size_t i;
    uint8_t c;
    float ce, qv, nb[6];
};

template <typename T>
__device__ __forceinline__ void fix_load(const StepArgs &a, const T *pn, size_t i, FixVox<T> &v)
{
    using IO = Io<T>;
    const size_t sy = a.px, sz = (size_t)a.px * a.ny;
    const T *P = static_cast<const T *>(a.p);
    v.i = i;
    v.c = __ldg(a.code + i);
    v.ce = IO::get(P[i]);
    v.qv = IO::get(pn[i]);
    v.nb[0] = IO::get(P[i + 1]);
    v.nb[1] = IO::get(P[i - 1]);
    v.nb[2] = IO::get(P[i + sy]);
    v.nb[3] = IO::get(P[i - sy]);
    v.nb[4] = IO::get(P[i + sz]);
    v.nb[5] = IO::get(P[i - sz]);
}

template <typename T> __device__ __forceinline__ void fix_store(const StepArgs &a, const FixVox<T> &v)
{
    const float r = leapfrog(v.c, v.ce, v.nb[0], v.nb[1], v.nb[2], v.nb[3], v.nb[4], v.nb[5], v.qv, a.c2dt2, a.inv_h2);
    static_cast<T *>(a.q)[v.i] = Io<T>::put(r);
}

template <typename T, int MAXS>
__global__ void __launch_bounds__(BT) k_boundary_fix(const __grid_constant__ StepArgs a, const void *pn,
                                                     const uint32_t *__restrict list, uint32_t nlist, uint32_t gb)
{
    if (a.stop && *a.stop) return;
    if (blockIdx.x < gb) {
        const uint64_t s0 = (uint64_t)blockIdx.x * BT + threadIdx.x;
        if (s0 >= a.nb) return;
        BVox<T, MAXS> v;
        bvox_load<T, BND_UPDATE, MAXS>(a, s0, v);
        bvox_update<T, BND_UPDATE, MAXS>(a, s0, v);
        return;
    }
    const uint32_t f0 = (blockIdx.x - gb) * BT + threadIdx.x;
    if (f0 >= nlist) return;
    FixVox<T> v;
    fix_load<T>(a, static_cast<const T *>(pn), __ldg(list + f0), v);
    fix_store<T>(a, v);
}

// batched: slot g belongs to the last member whose first boundary index is
// <= g (members without boundary voxels are skipped by that rule).  A
// block's 256 slots nearly always belong to one member: two threads find
// the members of the block's first and last slot (binary searches over the
// members' first indices), and when they agree the block copies that
// member's step arguments into shared memory once, so that no thread
// searches or reads its arguments from the descriptor array; a block that
// straddles members searches per thread between the two.
__device__ __forceinline__ uint32_t batch_member_of(const BatchMember *__restrict mem, uint32_t lo, uint32_t hi,
                                                    uint64_t g)
{
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) / 2;
        if (mem[mid].first_bnd <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename T, int MAXS>
__global__ void __launch_bounds__(256) k_boundary_batch(const BatchMember *__restrict mem, uint32_t nmem,
                                                        uint64_t ntotal, int parity)
{
    __shared__ StepArgs sa;
    __shared__ uint32_t sm[2];
    __shared__ uint64_t sfirst;
    const uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x, g = g0 + threadIdx.x;
    if (threadIdx.x < 2) {
        const uint64_t last = min(g0 + blockDim.x, ntotal) - 1;
        sm[threadIdx.x] = batch_member_of(mem, 0, nmem - 1, threadIdx.x == 0 ? g0 : last);
    }
    __syncthreads();
    const uint32_t m0 = sm[0], m1 = sm[1];
    if (m0 == m1) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(&mem[m0].step[parity]);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&sa);
        for (uint32_t k = threadIdx.x; k < (uint32_t)(sizeof(StepArgs) / 4); k += blockDim.x) dst[k] = src[k];
        if (threadIdx.x == 0) sfirst = mem[m0].first_bnd;
        __syncthreads();
        if (g >= ntotal) return;
        BVox<T, MAXS> v;
        bvox_load<T, BND_UPDATE, MAXS>(sa, g - sfirst, v);
        bvox_update<T, BND_UPDATE, MAXS>(sa, g - sfirst, v);
        return;
    }
    if (g >= ntotal) return;
    const BatchMember &b = mem[batch_member_of(mem, m0, m1, g)];
    BVox<T, MAXS> v;
    bvox_load<T, BND_UPDATE, MAXS>(b.step[parity], g - b.first_bnd, v);
    bvox_update<T, BND_UPDATE, MAXS>(b.step[parity], g - b.first_bnd, v);
}

// The reference's stop rule (simulator_gpu.cu:303-330) on receiver 0's
// samples of the steps before step sn, in the host rule's float operations
// and order: after step 3000 the RMS of the last 100 samples, through a
// slow first-order filter from step 3002 on; below 0.0009 the run stops.
__device__ __forceinline__ void stop_rule(const PostArgs &a, uint32_t sn)
{
    constexpr uint32_t RMS_SIZE = 100, MIN_RMS_CHECK_STEP = 3000;
    if (sn <= MIN_RMS_CHECK_STEP) return;
    float sum = 0.f;
    for (uint32_t i = sn - RMS_SIZE; i < sn; ++i) sum = __fadd_rn(sum, __fmul_rn(a.ir[i], a.ir[i]));
    float rms = __fsqrt_rn(__fdiv_rn(sum, (float)RMS_SIZE));
    float state = __uint_as_float(a.stop[2]);
    if (sn == MIN_RMS_CHECK_STEP + 1) {
        state = rms;
    } else {
        const float g = 0.00008f;
        const float vout = __fdiv_rn(__fadd_rn(__fmul_rn(g, rms), state), __fadd_rn(g, 1.f));
        state = __fsub_rn(__fmul_rn(2.f, vout), state);
        rms = vout;
    }
    a.stop[2] = __float_as_uint(state);
    if (rms < 0.0009f) {
        a.stop[1] = sn;
        a.stop[0] = 1u;
    }
}

template <typename T> __device__ __forceinline__ void post_body(const PostArgs &a)
{
    using IO = Io<T>;
    T *Q = static_cast<T *>(a.q);
    if (a.stop && a.stop[0]) return; // the stop rule fired at an earlier step
    const uint32_t sn = *a.ctr;
    // hard-source voxels (flag 3, simulator_gpu.cu:59-63): the stencils leave
    // them alone; their value of this step is written here, before the soft
    // sources are added
    if (a.nhpos) {
        // the step's own store at these voxels (phase 0 of the rounding key)
        const float hv = sn < a.nhard ? a.hard[sn] : 0.f;
        const uint32_t k0 = a.sr ? sr_step_key(sn, 0u) : 0u;
        for (uint32_t i = threadIdx.x; i < a.nhpos; i += blockDim.x)
            Q[a.hpos[i]] = put_rounded<T>(hv, a.sr, a.hpos[i], a.sr_base, k0);
        __syncthreads();
    }
    const uint32_t k1 = a.sr ? sr_step_key(sn, 1u) : 0u;
    for (uint32_t i = threadIdx.x; i < a.nsrc; i += blockDim.x) {
        const float v = sn < a.siglen ? a.sig[(uint64_t)i * a.siglen + sn] : 0.f;
        const uint64_t j = a.src[i];
        Q[j] = put_rounded<T>(__fadd_rn(IO::get(Q[j]), v), a.sr, j, a.sr_base, k1);
    }
    __syncthreads();
    if (sn < a.cap)
        for (uint32_t r = threadIdx.x; r < a.nrcv; r += blockDim.x)
            a.ir[(uint64_t)r * a.cap + sn] = __fmul_rn(IO::get(Q[a.rcv[r]]), a.inv_scale);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (a.stop && a.nrcv && sn < a.cap) stop_rule(a, sn);
        *a.ctr = sn + 1;
    }
}

template <typename T> __global__ void k_post(const __grid_constant__ PostArgs a) { post_body<T>(a); }

template <typename T> __global__ void k_post_batch(const BatchMember *__restrict mem, int parity)
{
    post_body<T>(mem[blockIdx.x].post[parity]);
}

template <typename T>
cudaError_t launch_step_t(int tile_rows, const StepArgs &a, cudaStream_t s)
{
    constexpr int TX = 32 * Io<T>::VEC;
    if (a.nz < 3 || a.ny < 3 || a.nx < 3) return cudaSuccess;
    const int zc = a.zc > 0 ? a.zc : default_planes(a.nz);
    StepArgs b = a;
    b.zc = zc;
    const unsigned gx = (a.px + TX - 1) / TX;
    if (a.ze <= a.zb) return cudaSuccess;
    const unsigned gz = (unsigned)((a.ze - a.zb + zc - 1) / zc);
    switch (tile_rows) {
    case 4: k_step<T, 4><<<dim3(gx, (a.ny + 3) / 4, gz), dim3(32, 4), 0, s>>>(b); break;
    case 16: k_step<T, 16><<<dim3(gx, (a.ny + 15) / 16, gz), dim3(32, 16), 0, s>>>(b); break;
    default: k_step<T, 8><<<dim3(gx, (a.ny + 7) / 8, gz), dim3(32, 8), 0, s>>>(b); break;
    }
    return cudaGetLastError();
}

} // namespace

int default_planes(uint32_t nz)
{
    (void)nz;
    return 32;
}

cudaError_t launch_step(int storage, int tile_rows, const StepArgs &a, cudaStream_t s)
{
    switch (storage) {
    case VIRS_STORAGE_F16: return launch_step_t<__half>(tile_rows, a, s);
    case VIRS_STORAGE_BF16: return launch_step_t<__nv_bfloat16>(tile_rows, a, s);
    default: return launch_step_t<float>(tile_rows, a, s);
    }
}

namespace {

template <typename T, int MODE>
void boundary_by_sections(uint32_t ns, unsigned g, const StepArgs &a, cudaStream_t s)
{
    if (MODE == BND_RECORD || ns <= 1) k_boundary<T, MODE, 1><<<g, BT, 0, s>>>(a);
    else if (ns == 2) k_boundary<T, MODE, 2><<<g, BT, 0, s>>>(a);
    else if (ns <= 4) k_boundary<T, MODE, 4><<<g, BT, 0, s>>>(a);
    else k_boundary<T, MODE, 0><<<g, BT, 0, s>>>(a);
}

template <typename T> void boundary_by_mode(int mode, uint32_t ns, unsigned g, const StepArgs &a, cudaStream_t s)
{
    switch (mode) {
    case BND_KEEP: boundary_by_sections<T, BND_KEEP>(ns, g, a, s); break;
    case BND_RECORD: boundary_by_sections<T, BND_RECORD>(ns, g, a, s); break;
    default: boundary_by_sections<T, BND_UPDATE>(ns, g, a, s); break;
    }
}

template <typename T>
void boundary_batch_by_sections(uint32_t maxs, unsigned g, const BatchMember *mem, uint32_t nmem, uint64_t nbnd,
                                int parity, cudaStream_t s)
{
    if (maxs <= 4) k_boundary_batch<T, 4><<<g, 256, 0, s>>>(mem, nmem, nbnd, parity);
    else k_boundary_batch<T, 0><<<g, 256, 0, s>>>(mem, nmem, nbnd, parity);
}

} // namespace

namespace {
template <typename T>
void boundary_fix_t(const StepArgs &a, const void *pn, const uint32_t *list, uint32_t nlist, cudaStream_t s)
{
    const unsigned gb = (unsigned)((a.nb + BT - 1) / BT);
    const unsigned g = gb + (nlist + BT - 1) / BT;
    const uint32_t ns = a.nsec;
    if (ns <= 1) k_boundary_fix<T, 1><<<g, BT, 0, s>>>(a, pn, list, nlist, gb);
    else if (ns == 2) k_boundary_fix<T, 2><<<g, BT, 0, s>>>(a, pn, list, nlist, gb);
    else if (ns <= 4) k_boundary_fix<T, 4><<<g, BT, 0, s>>>(a, pn, list, nlist, gb);
    else k_boundary_fix<T, 0><<<g, BT, 0, s>>>(a, pn, list, nlist, gb);
}
} // namespace

cudaError_t launch_boundary_fix(int storage, const StepArgs &a, const void *pn, const uint32_t *list, uint32_t nlist,
                                cudaStream_t s)
{
    if (a.nb == 0 && nlist == 0) return cudaSuccess;
    switch (storage) {
    case VIRS_STORAGE_F16: boundary_fix_t<__half>(a, pn, list, nlist, s); break;
    case VIRS_STORAGE_BF16: boundary_fix_t<__nv_bfloat16>(a, pn, list, nlist, s); break;
    default: boundary_fix_t<float>(a, pn, list, nlist, s); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_boundary(int storage, const StepArgs &a, int mode, cudaStream_t s)
{
    if (a.nb == 0) return cudaSuccess;
    const unsigned g = (unsigned)((a.nb + BT - 1) / BT);
    switch (storage) {
    case VIRS_STORAGE_F16: boundary_by_mode<__half>(mode, a.nsec, g, a, s); break;
    case VIRS_STORAGE_BF16: boundary_by_mode<__nv_bfloat16>(mode, a.nsec, g, a, s); break;
    default: boundary_by_mode<float>(mode, a.nsec, g, a, s); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_boundary_batch(int storage, const BatchMember *mem, uint32_t nmem, uint64_t nbnd, int parity,
                                  uint32_t max_sections, cudaStream_t s)
{
    if (nbnd == 0) return cudaSuccess;
    const unsigned g = (unsigned)((nbnd + 255) / 256);
    switch (storage) {
    case VIRS_STORAGE_F16: boundary_batch_by_sections<__half>(max_sections, g, mem, nmem, nbnd, parity, s); break;
    case VIRS_STORAGE_BF16:
        boundary_batch_by_sections<__nv_bfloat16>(max_sections, g, mem, nmem, nbnd, parity, s);
        break;
    default: boundary_batch_by_sections<float>(max_sections, g, mem, nmem, nbnd, parity, s); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_post_batch(int storage, const BatchMember *mem, uint32_t nmem, int parity, cudaStream_t s)
{
    switch (storage) {
    case VIRS_STORAGE_F16: k_post_batch<__half><<<nmem, 256, 0, s>>>(mem, parity); break;
    case VIRS_STORAGE_BF16: k_post_batch<__nv_bfloat16><<<nmem, 256, 0, s>>>(mem, parity); break;
    default: k_post_batch<float><<<nmem, 256, 0, s>>>(mem, parity); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_post(int storage, const PostArgs &a, cudaStream_t s)
{
    switch (storage) {
    case VIRS_STORAGE_F16: k_post<__half><<<1, 256, 0, s>>>(a); break;
    case VIRS_STORAGE_BF16: k_post<__nv_bfloat16><<<1, 256, 0, s>>>(a); break;
    default: k_post<float><<<1, 256, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

} // namespace virs
