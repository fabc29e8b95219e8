// The FDTD step with TMA-staged planes (the default kernel).
//
// Same arithmetic as kernels_step.cu (bit-identical results); the data path
// differs: a block owns a TX x TY tile of (x, y) and streams it along z, and
// every input plane reaches shared memory through the Tensor Memory
// Accelerator instead of through registers:
//   stage j holds  P(k+1)  the pressure plane above, with a one-voxel halo in
//                          y and a 16-byte halo in x   (TY+2) x (TX+2*PAD)
//                  Q(k)    p^{n-1} of the tile          TY x TX
//                  C(k)    the cell codes of the tile    TY x TX bytes
// for plane k = z0 - 2 + j.  The ring has D = L + 3 stages: planes z-1, z
// and z+1 are in use while L more are in flight, each stage guarded by one
// mbarrier that the TMA completes (complete_tx).  One thread issues the
// copies; after the block-wide barrier that ends the use of a stage it is
// refilled with the plane L+3 further on.  Out-of-range boxes (the y halo
// above row 0 or below the last row, x past the padded row) are zero-filled
// by the TMA.  Results go straight from registers to global memory with
// streaming 16-byte stores.  No multicast: every copy reads this GPU's own
// memory into this block's shared memory.
//
// Boundary voxels (flag 2): their leapfrog value is computed here with the
// staged neighbours and written, with p and p^{n-1}, to the voxel's slot of
// the compacted boundary list; p^{n-1} stays in place.  The boundary pass
// (k_boundary) then applies the filters to those records, coalesced, so the
// only divergent work here is one warp scan and one 16-byte store per
// boundary voxel.
//
// Every wait on an mbarrier is bounded; a wait that gives up sets *err and
// the block returns (the host turns that into VIRS_E_TIMEOUT).
#include <cuda.h>

#include <algorithm>

#include "step_common.cuh"

namespace virs {
namespace {

using namespace step;

constexpr unsigned FULL = 0xffffffffu;
constexpr int TX = 128;
// A waiting thread asks to be parked for up to WAIT_HINT_NS per try (it
// resumes as soon as the stage's phase completes), so the waiting warp does
// not spin on issue slots that the computing warps need; the whole wait is
// bounded by WAIT_LIMIT_NS of the global timer.
constexpr uint32_t WAIT_HINT_NS = 20000;
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(saddr(b)), "r"(parity), "r"(WAIT_HINT_NS)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
                 ::"r"(saddr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(saddr(bar)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}

template <typename T> struct Geo {
    static constexpr int PAD = 16 / (int)sizeof(T); // x halo: one 16-byte chunk on each side
    static constexpr int PW = TX + 2 * PAD;
};

template <typename T, int TY> struct Stage {
    static constexpr uint32_t PB = Geo<T>::PW * (TY + 2) * sizeof(T);
    static constexpr uint32_t QB = TX * TY * sizeof(T);
    static constexpr uint32_t CB = TX * TY;
    static constexpr uint32_t BB = 4 * TY * sizeof(uint32_t); // 4 prefix segments per tile row
    static constexpr uint32_t PBa = (PB + 127u) & ~127u;
    static constexpr uint32_t QBa = (QB + 127u) & ~127u;
    static constexpr uint32_t CBa = (CB + 127u) & ~127u;
    static constexpr uint32_t BBa = (BB + 127u) & ~127u;
    static constexpr uint32_t SB = PBa + QBa + CBa + BBa;
};

template <typename T> __device__ __forceinline__ void ld4(const T *p, float (&r)[4]);
template <> __device__ __forceinline__ void ld4<float>(const float *p, float (&r)[4])
{
    const float4 v = *reinterpret_cast<const float4 *>(p);
    r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
}
template <> __device__ __forceinline__ void ld4<__half>(const __half *p, float (&r)[4])
{
    const uint2 v = *reinterpret_cast<const uint2 *>(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&v.y));
    r[0] = a.x; r[1] = a.y; r[2] = b.x; r[3] = b.y;
}
template <> __device__ __forceinline__ void ld4<__nv_bfloat16>(const __nv_bfloat16 *p, float (&r)[4])
{
    const uint2 v = *reinterpret_cast<const uint2 *>(p);
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&v.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&v.y));
    r[0] = a.x; r[1] = a.y; r[2] = b.x; r[3] = b.y;
}

template <typename T> __device__ __forceinline__ void st4(T *p, const float (&r)[4]);
template <> __device__ __forceinline__ void st4<float>(float *p, const float (&r)[4])
{
    __stcs(reinterpret_cast<float4 *>(p), make_float4(r[0], r[1], r[2], r[3]));
}
template <> __device__ __forceinline__ void st4<__half>(__half *p, const float (&r)[4])
{
    uint2 v;
    *reinterpret_cast<__half2 *>(&v.x) = __floats2half2_rn(r[0], r[1]);
    *reinterpret_cast<__half2 *>(&v.y) = __floats2half2_rn(r[2], r[3]);
    __stcs(reinterpret_cast<uint2 *>(p), v);
}
template <> __device__ __forceinline__ void st4<__nv_bfloat16>(__nv_bfloat16 *p, const float (&r)[4])
{
    uint2 v;
    *reinterpret_cast<__nv_bfloat162 *>(&v.x) = __floats2bfloat162_rn(r[0], r[1]);
    *reinterpret_cast<__nv_bfloat162 *>(&v.y) = __floats2bfloat162_rn(r[2], r[3]);
    __stcs(reinterpret_cast<uint2 *>(p), v);
}

// waits for phase `parity` of *b for at most limit_ns; on timeout sets *err
__device__ __forceinline__ bool bounded_wait(uint64_t *b, uint32_t parity, uint64_t limit_ns, int *err)
{
    if (mbar_try_wait_hint(b, parity)) return true;
    const uint64_t t0 = global_ns();
    do {
        if (mbar_try_wait_hint(b, parity)) return true;
    } while (global_ns() - t0 < limit_ns);
    atomicExch(err, 1);
    return false;
}

__device__ __forceinline__ bool wait_stage(uint64_t *bars, int j, int D, int *err)
{
    return bounded_wait(bars + (j % D), (uint32_t)((j / D) & 1), WAIT_LIMIT_NS, err);
}

// One tile (bx, by, bz) of one simulation.  `jg` is the block's running
// count of issued stages; it continues across tiles so that the ring slot
// and mbarrier phase of every stage stay consistent when a block processes
// several tiles (the batched kernel).  Returns false when a bounded wait
// gave up.
template <typename T, int TY, int L>
__device__ __forceinline__ bool step_tile(const StepArgs &a, const CUtensorMap *mP, const CUtensorMap *mQ,
                                          const CUtensorMap *mC, const CUtensorMap *mB, int bx, int by, int bz,
                                          int *err, unsigned char *smem, uint64_t *bars, uint32_t &jg)
{
    using S = Stage<T, TY>;
    constexpr int PAD = Geo<T>::PAD, PW = Geo<T>::PW;
    constexpr int D = L + 3;

    const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;
    const int x0 = bx * TX;
    const int x = x0 + lane * 4;
    const int y0 = by * TY;
    const int y = y0 + ty;
    const int z0 = 1 + bz * a.zc;
    const int z1 = min(z0 + a.zc, (int)a.nz - 1);
    if (z0 >= z1) return true;
    const int jmax = z1 - z0 + 1; // last stage ordinal (plane z1 - 1)
    const int ny = (int)a.ny;
    const bool act = x < (int)a.px && y < ny;
    const size_t plane = (size_t)a.px * ny;
    T *Q = static_cast<T *>(a.q);
    const uint32_t j0 = jg;
    const int seg = x0 / SEG, seg4 = seg & ~3; // prefix box starts on a 16-byte boundary

    auto issue = [&](int j) {
        const int k = z0 - 2 + j;
        const uint32_t g = j0 + (uint32_t)j;
        unsigned char *st = smem + (g % D) * S::SB;
        uint64_t *b = bars + (g % D);
        const bool full = j >= 2;
        mbar_expect_tx(b, S::PB + (full ? S::QB + S::CB + S::BB : 0u));
        tma_load_3d(st, mP, b, x0 - PAD, y0 - 1, k + 1);
        if (full) {
            tma_load_3d(st + S::PBa, mQ, b, x0, y0, k);
            tma_load_3d(st + S::PBa + S::QBa, mC, b, x0, y0, k);
            tma_load_3d(st + S::PBa + S::QBa + S::CBa, mB, b, seg4, y0, k);
        }
    };
    if (tid == 0)
        for (int j = 0; j < D && j <= jmax; ++j) issue(j);

    for (int i = 0, z = z0; z < z1; ++i, ++z) {
        // thread 0 waits for the stage (bounded); the barrier then tells every
        // thread that the stage is ready and that everyone is done with plane
        // z-1, so the stage that held P(z-2) can be refilled
        bool bad = false;
        if (tid == 0) {
            bad = !wait_stage(bars, j0 + i + 2, D, err);
            if (i == 0) bad = bad || !wait_stage(bars, j0, D, err) || !wait_stage(bars, j0 + 1, D, err);
        }
        if (__syncthreads_or(bad)) return false;
        if (tid == 0 && i >= 1 && i + L + 2 <= jmax) issue(i + L + 2);

        const T *Pm = reinterpret_cast<const T *>(smem + ((j0 + i) % D) * S::SB);       // P(z-1)
        const T *Pc = reinterpret_cast<const T *>(smem + ((j0 + i + 1) % D) * S::SB);   // P(z)
        const unsigned char *s2 = smem + ((j0 + i + 2) % D) * S::SB;
        const T *Pp = reinterpret_cast<const T *>(s2);                                   // P(z+1)
        const T *Qs = reinterpret_cast<const T *>(s2 + S::PBa);
        const uint32_t code4 = *reinterpret_cast<const uint32_t *>(s2 + S::PBa + S::QBa + ty * TX + lane * 4);

        const int c0 = (ty + 1) * PW + PAD + lane * 4;
        float cc[4], ym[4], yp[4], zm[4], zp[4], qv[4];
        ld4(Pc + c0, cc);
        ld4(Pc + c0 - PW, ym);
        ld4(Pc + c0 + PW, yp);
        ld4(Pm + c0, zm);
        ld4(Pp + c0, zp);
        ld4(Qs + ty * TX + lane * 4, qv);
        float left = __shfl_up_sync(FULL, cc[3], 1);
        float right = __shfl_down_sync(FULL, cc[0], 1);
        if (lane == 0) left = Io<T>::get(Pc[c0 - 1]);
        if (lane == 31) right = Io<T>::get(Pc[c0 + 4]);

        float r[4];
        unsigned bmask = 0;
        if (code4 == 0u) {
            // four air voxels without wall neighbours: the common case
            r[0] = leapfrog_air(cc[0], cc[1], left, yp[0], ym[0], zp[0], zm[0], qv[0], a.c2dt2, a.inv_h2);
            r[1] = leapfrog_air(cc[1], cc[2], cc[0], yp[1], ym[1], zp[1], zm[1], qv[1], a.c2dt2, a.inv_h2);
            r[2] = leapfrog_air(cc[2], cc[3], cc[1], yp[2], ym[2], zp[2], zm[2], qv[2], a.c2dt2, a.inv_h2);
            r[3] = leapfrog_air(cc[3], right, cc[2], yp[3], ym[3], zp[3], zm[3], qv[3], a.c2dt2, a.inv_h2);
        } else
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint8_t c = (uint8_t)(code4 >> (8 * k));
            const float xm = k == 0 ? left : cc[k - 1];
            const float xp = k == 3 ? right : cc[k + 1];
            if (c >= CODE_HARD) {
                if (c == CODE_NONE) r[k] = qv[k];
                else if (c == CODE_WALL) r[k] = 0.f;
                else {
                    const uint32_t sn = __ldg(a.ctr);
                    r[k] = sn < a.nhard ? __ldg(a.hard + sn) : 0.f;
                }
            } else {
                r[k] = leapfrog(c, cc[k], xp, xm, yp[k], ym[k], zp[k], zm[k], qv[k], a.c2dt2, a.inv_h2);
                if (c & CODE_BND) bmask |= 1u << k;
            }
        }
        // Boundary voxels: the record {free value, p, p^{n-1}} goes to their
        // slot of the compacted list for the boundary pass, and p^{n-1} stays
        // in place.  A warp covers consecutive voxels of one row, so the slot
        // is the row segment's prefix (staged with the plane) plus a warp scan.
        if (!act) bmask = 0;
        if (__any_sync(FULL, bmask != 0)) {
            const int cnt = __popc(bmask);
            int inc = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULL, inc, o);
                if (lane >= o) inc += t;
            }
            if (bmask) {
                const uint32_t *bs = reinterpret_cast<const uint32_t *>(s2 + S::PBa + S::QBa + S::CBa);
                uint64_t slot = (uint64_t)bs[ty * 4 + (seg - seg4)] + (uint64_t)(inc - cnt);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (bmask & (1u << k)) {
                        a.side[slot++] = make_float4(r[k], cc[k], qv[k], 0.f);
                        r[k] = qv[k];
                    }
            }
        }
        if (act) st4(Q + (size_t)z * plane + (size_t)y * a.px + x, r);
    }
    jg = j0 + (uint32_t)jmax + 1;
    return true;
}

template <int D> __device__ __forceinline__ void init_bars(uint64_t *bars)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int s = 0; s < D; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

template <typename T, int TY, int L>
__global__ void __launch_bounds__(32 * TY, 1024 / (32 * TY)) k_step_tma(const __grid_constant__ StepArgs a,
                                                                        const __grid_constant__ CUtensorMap mP,
                                                                        const __grid_constant__ CUtensorMap mQ,
                                                                        const __grid_constant__ CUtensorMap mC,
                                                                        const __grid_constant__ CUtensorMap mB, int *err)
{
    constexpr int D = L + 3;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + D * Stage<T, TY>::SB);
    init_bars<D>(bars);
    uint32_t jg = 0;
    step_tile<T, TY, L>(a, &mP, &mQ, &mC, &mB, blockIdx.x, blockIdx.y, blockIdx.z, err, smem, bars, jg);
}

// Many simulations in one launch: the blocks walk the concatenated tile
// lists of all members (tiles of a member are consecutive, so neighbouring
// tiles run at the same time and share the halo rows in L2), either one
// tile per block or, persistent, a single wave of blocks striding over all.
template <typename T, int TY, int L>
__global__ void __launch_bounds__(32 * TY, 1024 / (32 * TY)) k_step_tma_batch(const BatchMember *__restrict mem,
                                                                              uint32_t nmem, uint64_t ntiles,
                                                                              int parity, int *err)
{
    constexpr int D = L + 3;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + D * Stage<T, TY>::SB);
    init_bars<D>(bars);
    uint32_t jg = 0;
    uint32_t m = 0;
    for (uint64_t w = blockIdx.x; w < ntiles; w += gridDim.x) {
        while (m + 1 < nmem && mem[m + 1].first_tile <= w) ++m;   // tiles are visited in increasing order
        const BatchMember &b = mem[m];
        const uint64_t local = w - b.first_tile;
        const int bx = (int)(local % b.gx), by = (int)((local / b.gx) % b.gy), bz = (int)(local / ((uint64_t)b.gx * b.gy));
        __syncthreads(); // every thread is done with the previous tile's stages
        if (!step_tile<T, TY, L>(b.step[parity], &b.mapP[parity], &b.mapQ[parity ^ 1], &b.mapC, &b.mapB, bx, by, bz,
                                 err, smem, bars, jg))
            return;
    }
}

template <typename T, int TY, int L> constexpr size_t smem_bytes()
{
    return (size_t)(L + 3) * Stage<T, TY>::SB + (L + 3) * sizeof(uint64_t);
}

template <typename T, int TY, int L>
cudaError_t launch3(const StepArgs &a, const TmaMaps &m, int *err, cudaStream_t s)
{
    auto kern = k_step_tma<T, TY, L>;
    constexpr size_t sm = smem_bytes<T, TY, L>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const unsigned gx = (a.px + TX - 1) / TX;
    const unsigned gz = (a.nz - 2 + a.zc - 1) / a.zc;
    kern<<<dim3(gx, (a.ny + TY - 1) / TY, gz), dim3(32, TY), sm, s>>>(a, *m.p, *m.q, *m.c, *m.b, err);
    return cudaGetLastError();
}

template <typename T, int TY>
cudaError_t launch2(int depth, const StepArgs &a, const TmaMaps &m, int *err, cudaStream_t s)
{
    switch (depth) {
    case 1: return launch3<T, TY, 1>(a, m, err, s);
    case 3: return launch3<T, TY, 3>(a, m, err, s);
    default: return launch3<T, TY, 2>(a, m, err, s);
    }
}

template <typename T>
cudaError_t launch1(int rows, int depth, const StepArgs &a, const TmaMaps &m, int *err, cudaStream_t s)
{
    switch (rows) {
    case 4: return launch2<T, 4>(depth, a, m, err, s);
    case 16: return launch2<T, 16>(depth, a, m, err, s);
    default: return launch2<T, 8>(depth, a, m, err, s);
    }
}

// Waits on an mbarrier that nothing completes, for limit_us microseconds,
// with the bounded wait of the step kernels, which reports the timeout
// through *err.
__global__ void k_wait_probe(int *err, uint32_t limit_us)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) bounded_wait(&bar, 0, (uint64_t)limit_us * 1000ull, err);
}

template <typename T, int TY, int L>
cudaError_t launch_batch3(const BatchMember *mem, uint32_t nmem, uint64_t ntiles, int parity, bool persistent, int *err,
                          cudaStream_t s)
{
    auto kern = k_step_tma_batch<T, TY, L>;
    constexpr size_t sm = smem_bytes<T, TY, L>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, per = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 32 * TY, sm)) != cudaSuccess) return e;
    // persistent: one wave of blocks walks all tiles; otherwise one block per
    // tile and the hardware scheduler overlaps the blocks' prologues
    const uint64_t cap = persistent ? (uint64_t)nsm * (uint64_t)std::max(per, 1) : (uint64_t)INT32_MAX;
    const uint64_t grid = std::min<uint64_t>(ntiles, cap);
    kern<<<(unsigned)grid, dim3(32, TY), sm, s>>>(mem, nmem, ntiles, parity, err);
    return cudaGetLastError();
}

template <typename T, int TY>
cudaError_t launch_batch2(int depth, const BatchMember *mem, uint32_t nmem, uint64_t ntiles, int parity,
                          bool persistent, int *err, cudaStream_t s)
{
    switch (depth) {
    case 1: return launch_batch3<T, TY, 1>(mem, nmem, ntiles, parity, persistent, err, s);
    case 3: return launch_batch3<T, TY, 3>(mem, nmem, ntiles, parity, persistent, err, s);
    default: return launch_batch3<T, TY, 2>(mem, nmem, ntiles, parity, persistent, err, s);
    }
}

template <typename T>
cudaError_t launch_batch1(int rows, int depth, const BatchMember *mem, uint32_t nmem, uint64_t ntiles, int parity,
                          bool persistent, int *err, cudaStream_t s)
{
    switch (rows) {
    case 4: return launch_batch2<T, 4>(depth, mem, nmem, ntiles, parity, persistent, err, s);
    case 16: return launch_batch2<T, 16>(depth, mem, nmem, ntiles, parity, persistent, err, s);
    default: return launch_batch2<T, 8>(depth, mem, nmem, ntiles, parity, persistent, err, s);
    }
}

} // namespace

cudaError_t launch_step_tma_batch(int storage, int tile_rows, int depth, const BatchMember *mem, uint32_t nmem,
                                  uint64_t ntiles, int parity, bool persistent, int *err, cudaStream_t s)
{
    if (ntiles == 0) return cudaSuccess;
    switch (storage) {
    case VIRS_STORAGE_F16:
        return launch_batch1<__half>(tile_rows, depth, mem, nmem, ntiles, parity, persistent, err, s);
    case VIRS_STORAGE_BF16:
        return launch_batch1<__nv_bfloat16>(tile_rows, depth, mem, nmem, ntiles, parity, persistent, err, s);
    default: return launch_batch1<float>(tile_rows, depth, mem, nmem, ntiles, parity, persistent, err, s);
    }
}

int tma_box_width(int storage) { return storage == VIRS_STORAGE_F32 ? TX + 8 : TX + 16; }
int tma_pad(int storage) { return storage == VIRS_STORAGE_F32 ? 4 : 8; }
int tma_tile_x() { return TX; }

cudaError_t launch_wait_probe(int *err, uint32_t limit, cudaStream_t s)
{
    k_wait_probe<<<1, 32, 0, s>>>(err, limit);
    return cudaGetLastError();
}

cudaError_t launch_step_tma(int storage, int tile_rows, int depth, const StepArgs &a0, const TmaMaps &m, int *err,
                            cudaStream_t s)
{
    if (a0.nz < 3 || a0.ny < 3 || a0.nx < 3) return cudaSuccess;
    StepArgs a = a0;
    if (a.zc <= 0) a.zc = default_planes(a.nz);
    switch (storage) {
    case VIRS_STORAGE_F16: return launch1<__half>(tile_rows, depth, a, m, err, s);
    case VIRS_STORAGE_BF16: return launch1<__nv_bfloat16>(tile_rows, depth, a, m, err, s);
    default: return launch1<float>(tile_rows, depth, a, m, err, s);
    }
}

} // namespace virs
