// The FDTD step with TMA-staged planes (the default kernel).
//
// Same arithmetic as kernels_step.cu (bit-identical results); the data path
// differs: a block owns a TX x TY tile of (x, y) and streams it along z, and
// every input plane reaches shared memory through the Tensor Memory
// Accelerator instead of through registers:
//   stage j holds  P(k)  the pressure plane k with a one-voxel halo in y and
//                        a 16-byte halo in x      (TY+2) x (TX+2*PAD)
//                  Q(k)  p^{n-1} of the tile       TY x TX
//                  C(k)  the cell codes of the tile TY x TX bytes
// for plane k = z0 - 1 + j.  A plane of a tile whose codes are all zero
// (plain air: most of a large room's interior) is marked in the tile's
// 64-bit mask (a.tzmask, built per tiling at set-up); its codes are not
// copied and every voxel takes the air update.  Each thread updates the V
// voxels of one
// 16-byte vector; the centres of P(z-1) and P(z) stay in its registers, so
// the ring has D = L + 2 stages: planes z and z+1 are in use while L more
// are in flight, each stage guarded by one mbarrier that the TMA completes
// (complete_tx).  One thread issues the copies; after the block-wide
// barrier that ends the use of a stage it is refilled with the plane D
// further on.  Out-of-range boxes (the y halo above row 0 or below the last
// row, x past the padded row) are zero-filled by the TMA.  Results go
// straight from registers to global memory with streaming 16-byte stores.
// No multicast: every copy reads this GPU's own memory into this block's
// shared memory.
//
// Every voxel is first updated as air without wall neighbours (packed FP32
// pairs).  Warps whose codes are not all zero then fix the other voxels
// with selects: border voxels and boundary voxels (flag 2) keep p^{n-1},
// walls take 0 and hard sources their value.  The boundary pass
// (k_boundary) updates the boundary voxels afterwards from the p^n buffer,
// which this kernel does not write.
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

// Thread layout: every thread updates V consecutive voxels of one row, the
// ones one 16-byte vector holds (4 FP32 or 8 16-bit values); a tile row is
// TX = 128 voxels, so LPR = 128 / V lanes share a row and a warp covers RPW
// rows (1 for FP32, 2 for 16-bit storage).
template <typename T> struct Lay {
    static constexpr int V = 16 / (int)sizeof(T);
    static constexpr int LPR = TX / V;
    static constexpr int RPW = 32 / LPR;
    static constexpr int PAD = 16 / (int)sizeof(T); // x halo: one 16-byte chunk on each side
    static constexpr int PW = TX + 2 * PAD;
};

template <typename T, int TY> struct Stage {
    static constexpr uint32_t PB = Lay<T>::PW * (TY + 2) * sizeof(T);
    static constexpr uint32_t QB = TX * TY * sizeof(T);
    static constexpr uint32_t CB = TX * TY;
    static constexpr uint32_t PBa = (PB + 127u) & ~127u;
    static constexpr uint32_t QBa = (QB + 127u) & ~127u;
    static constexpr uint32_t CBa = (CB + 127u) & ~127u;
    static constexpr uint32_t SB = PBa + QBa + CBa;
};

// the V cell codes of a thread (4 or 8 bytes)
template <int V> struct Codes;
// bytes with bit 7 clear and some other bit set: bit 7 of each byte of
// ((w & 0x7f..) + 0x7f..) & ~w
__device__ __forceinline__ uint32_t mirror_bytes(uint32_t w)
{
    return ((w & 0x7f7f7f7fu) + 0x7f7f7f7fu) & ~w & 0x80808080u;
}
template <> struct Codes<4> {
    uint32_t w;
    __device__ void load(const unsigned char *p) { w = *reinterpret_cast<const uint32_t *>(p); }
    __device__ void clear() { w = 0u; }
    __device__ bool any() const { return w != 0u; }
    __device__ uint32_t get(int k) const { return (w >> (8 * k)) & 0xffu; }
    __device__ uint32_t mirror() const { return mirror_bytes(w); }
    __device__ bool is_mirror(uint32_t m, int k) const { return (m >> (8 * k + 7)) & 1u; }
};
template <> struct Codes<8> {
    uint2 w;
    __device__ void load(const unsigned char *p) { w = *reinterpret_cast<const uint2 *>(p); }
    __device__ void clear() { w = make_uint2(0u, 0u); }
    __device__ bool any() const { return (w.x | w.y) != 0u; }
    __device__ uint32_t get(int k) const { return ((k < 4 ? w.x : w.y) >> (8 * (k & 3))) & 0xffu; }
    // the mirror bytes of the two words folded into one: bit 7 of byte k
    // (k < 4) from w.x, bit 6 of byte k - 4 from w.y
    __device__ uint32_t mirror() const { return mirror_bytes(w.x) | (mirror_bytes(w.y) >> 1); }
    __device__ bool is_mirror(uint32_t m, int k) const { return (m >> (8 * (k & 3) + (k < 4 ? 7 : 6))) & 1u; }
};

// The update of one thread's V voxels of a plane: cc holds the centres,
// left / right the x neighbours beyond the vector, ym / yp / zm / zp the y
// and z neighbours, qv p^{n-1}.
template <typename T>
__device__ __forceinline__ void tile_update(const Codes<Lay<T>::V> &code, const float (&cc)[Lay<T>::V], float left,
                                        float right, const float (&yp)[Lay<T>::V], const float (&ym)[Lay<T>::V],
                                        const float (&zp)[Lay<T>::V], const float (&zm)[Lay<T>::V],
                                        const float (&qv)[Lay<T>::V], float2 c2dt2, float2 inv_h2, float c2dt2s,
                                        float inv_h2s, float (&r)[Lay<T>::V])
{
    constexpr int V = Lay<T>::V;
    // every voxel as air without wall neighbours, the common case, two
    // at a time ...
#pragma unroll
    for (int k = 0; k < V; k += 2) {
        const float2 x2 = make_float2(__fadd_rn(cc[k + 1], k > 0 ? cc[k - 1] : left),
                                      __fadd_rn(k + 2 < V ? cc[k + 2] : right, cc[k]));
        const float2 o = leapfrog_air2(make_float2(cc[k], cc[k + 1]), x2, make_float2(yp[k], yp[k + 1]),
                                       make_float2(ym[k], ym[k + 1]), make_float2(zp[k], zp[k + 1]),
                                       make_float2(zm[k], zm[k + 1]), make_float2(qv[k], qv[k + 1]), c2dt2, inv_h2);
        r[k] = o.x;
        r[k + 1] = o.y;
    }
    // ... then the voxels with another code.  Walls take 0; border,
    // hard-source and boundary voxels keep p^{n-1} (the post kernel
    // writes the hard-source value, the boundary pass updates boundary
    // voxels from the untouched p^n buffer): a test and a select per
    // voxel, no divergence.  Only air next to a wall outside the
    // boundary layer (a grid without a sponge layer) needs the update
    // with the mirror rule; such codes have bit 7 clear and other bits
    // set, found for four bytes at once.
    if (__any_sync(FULL, code.any())) {
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const uint32_t c = code.get(k);
            if (c & CODE_BND) r[k] = c == CODE_WALL ? 0.f : qv[k];
        }
        const uint32_t mirror = code.mirror();
        if (__any_sync(FULL, mirror != 0u)) {
#pragma unroll
            for (int k = 0; k < V; ++k)
                if (code.is_mirror(mirror, k))
                    r[k] = leapfrog((uint8_t)code.get(k), cc[k], k == V - 1 ? right : cc[k + 1],
                                    k == 0 ? left : cc[k - 1], yp[k], ym[k], zp[k], zm[k], qv[k], c2dt2s, inv_h2s);
        }
    }
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

__device__ __forceinline__ bool wait_stage(uint64_t *bars, uint32_t j, int D, int *err)
{
    return bounded_wait(bars + (j % D), (j / D) & 1u, WAIT_LIMIT_NS, err);
}

// The per-tile constants of the plane loop.  SR: the 16-bit stores round
// stochastically (a compile-time choice, so that the default path carries
// no trace of it).
template <typename T, int TY, int L, bool SR = false> struct Tile {
    const StepArgs *a;
    unsigned char *smem;
    uint64_t *bars;
    const CUtensorMap *mP, *mQ, *mC;
    int *err;
    int x0, y0, z0, nst, row, sl, c0, t0;
    uint32_t j0;
    bool act, leader;
    uint32_t srk; // the stochastic-rounding key of this step's stores (a->sr)
    float2 c2dt2, inv_h2;
    size_t plane;
    uint64_t zmask; // bit j: the codes of stage j are all zero (not copied)

    // the codes of stage j are all zero and not copied
    __device__ __forceinline__ bool codes_zero(int j) const { return j < 64 && ((zmask >> j) & 1ull); }

    static constexpr int D = L + 2;
    using S = Stage<T, TY>;

    // stage j holds plane z0 - 1 + j (see step_tile)
    __device__ __forceinline__ void issue(int j) const
    {
        constexpr int PAD = Lay<T>::PAD;
        const int k = z0 - 1 + j;
        const uint32_t g = j0 + (uint32_t)j;
        unsigned char *st = smem + (g % D) * S::SB;
        uint64_t *b = bars + (g % D);
        const bool full = j >= 1 && j <= nst - 2;
        const bool codes = full && !codes_zero(j);
        mbar_expect_tx(b, S::PB + (full ? S::QB : 0u) + (codes ? S::CB : 0u));
        tma_load_3d(st, mP, b, x0 - PAD, y0 - 1, k);
        if (full) tma_load_3d(st + S::PBa, mQ, b, x0, y0, k);
        if (codes) tma_load_3d(st + S::PBa + S::QBa, mC, b, x0, y0, k);
    }

    // Plane z = z0 + i: zm and cc hold the centres of P(z-1) and P(z); the
    // centre of P(z+1) is loaded into zp.  `sh` is the ring slot of the
    // stage of z, `out` the thread's first output voxel of plane z.
    __device__ __forceinline__ bool plane_step(int i, const float (&zm)[Lay<T>::V], const float (&cc)[Lay<T>::V],
                                               float (&zp)[Lay<T>::V], uint32_t &sh, T *&out) const
    {
        using IO = Io<T>;
        constexpr int V = Lay<T>::V, LPR = Lay<T>::LPR, PW = Lay<T>::PW;
        // the leader waits for the stage of z+1 (bounded); the barrier then
        // tells every thread that it is ready and that everyone is done with
        // the stage of z-1, which is refilled with the plane D on
        bool bad = false;
        if (leader) bad = !wait_stage(bars, j0 + (uint32_t)i + 2u, D, err);
        if (__syncthreads_or(bad)) return false;
        if (leader && i + D < nst) issue(i + D);
        const uint32_t sz = sh + 1u == (uint32_t)D ? 0u : sh + 1u;

        const unsigned char *s0 = smem + sh * S::SB;
        const T *Ph = reinterpret_cast<const T *>(s0);
        float ym[V], yp[V], qv[V];
        IO::ld(reinterpret_cast<const T *>(smem + sz * S::SB) + c0, zp);
        IO::ld(Ph + c0 - PW, ym);
        IO::ld(Ph + c0 + PW, yp);
        IO::ld(reinterpret_cast<const T *>(s0 + S::PBa) + t0, qv);
        Codes<V> code; // stage i + 1 holds plane z
        if (codes_zero(i + 1)) code.clear();
        else code.load(s0 + S::PBa + S::QBa + t0);
        float left = __shfl_up_sync(FULL, cc[V - 1], 1, LPR);
        float right = __shfl_down_sync(FULL, cc[0], 1, LPR);
        if (sl == 0) left = IO::ld1(Ph + c0 - 1);
        if (sl == LPR - 1) right = IO::ld1(Ph + c0 + V);

        float r[V];
        tile_update<T>(code, cc, left, right, yp, ym, zp, zm, qv, c2dt2, inv_h2, a->c2dt2, a->inv_h2, r);
        if (act) {
            if constexpr (SR) st_sr<T>(out, r, (uint64_t)(out - static_cast<T *>(a->q)), a->sr_base, srk);
            else IO::st(out, r);
        }
        out += plane;
        sh = sz;
        return true;
    }
};

// One tile (bx, by, bz) of one simulation.  Stage j of the tile holds the
// plane k = z0 - 1 + j: P(k) with its halo, and for k in [z0, z1) also Q(k)
// and the codes of plane k.  The
// centres of P(z-1) and P(z) stay in registers from the previous planes, so
// plane z reads the stage of z (halo neighbours, Q, codes) and the centre
// of the stage of z+1; the ring has D = L + 2 slots.  The plane loop is
// unrolled three times so that the three centre planes change roles
// without register copies.  `jg` is the block's running count of issued
// stages: it continues across tiles so that the ring slot and mbarrier
// phase of every stage stay consistent when a block processes several
// tiles (the batched kernel).  Returns false when a bounded wait gave up.
template <typename T, int TY, int L, bool SR>
__device__ __forceinline__ bool step_tile(const StepArgs &a, const CUtensorMap *mP, const CUtensorMap *mQ,
                                          const CUtensorMap *mC, int bx, int by, int bz, int *err, unsigned char *smem,
                                          uint64_t *bars, uint32_t &jg)
{
    using G = Lay<T>;
    using S = Stage<T, TY>;
    using IO = Io<T>;
    constexpr int V = G::V, LPR = G::LPR, PAD = G::PAD, PW = G::PW;
    constexpr int D = L + 2;
    static_assert(IO::VEC == V && V % 2 == 0, "one 16-byte vector per thread, an even number of voxels");

    Tile<T, TY, L, SR> t;
    const int lane = threadIdx.x, tid = threadIdx.y * 32 + lane;
    t.a = &a;
    t.smem = smem;
    t.bars = bars;
    t.mP = mP;
    t.mQ = mQ;
    t.mC = mC;
    t.err = err;
    t.row = threadIdx.y * G::RPW + lane / LPR; // row of the tile
    t.sl = lane % LPR;                         // lane within the row
    t.x0 = bx * TX;
    t.y0 = by * TY;
    t.z0 = a.zb + bz * a.zc;
    const int z1 = min(t.z0 + a.zc, a.ze);
    if (t.z0 >= z1) return true;
    t.nst = z1 - t.z0 + 2; // stages: planes z0-1 .. z1
    const int x = t.x0 + t.sl * V, y = t.y0 + t.row;
    t.act = x < (int)a.px && y < (int)a.ny;
    t.leader = tid == 0;
    t.j0 = jg;
    t.c0 = (t.row + 1) * PW + PAD + t.sl * V; // this thread's first voxel in a halo box
    t.t0 = t.row * TX + t.sl * V;            // ... and in a tile box
    t.c2dt2 = make_float2(a.c2dt2, a.c2dt2);
    t.inv_h2 = make_float2(a.inv_h2, a.inv_h2);
    t.srk = SR ? sr_step_key(*a.ctr, 0u) : 0u;
    t.plane = (size_t)a.px * a.ny;
    {
        const uint32_t gx = (a.px + TX - 1) / TX, gy = (a.ny + TY - 1) / TY;
        t.zmask = a.tzmask ? __ldg(a.tzmask + ((size_t)bz * gy + (size_t)by) * gx + (size_t)bx) : 0ull;
    }

    if (t.leader)
        for (int j = 0; j < D && j < t.nst; ++j) t.issue(j);

    float A[V], B[V], C[V];
    {
        bool bad = false;
        if (t.leader) bad = !wait_stage(bars, t.j0, D, err) || !wait_stage(bars, t.j0 + 1u, D, err);
        if (__syncthreads_or(bad)) return false;
        IO::ld(reinterpret_cast<const T *>(smem + (t.j0 % D) * S::SB) + t.c0, A);        // P(z0-1)
        IO::ld(reinterpret_cast<const T *>(smem + ((t.j0 + 1u) % D) * S::SB) + t.c0, B); // P(z0)
    }
    uint32_t sh = (t.j0 + 1u) % D; // slot of the stage of plane z
    T *out = static_cast<T *>(a.q) + ((size_t)t.z0 * a.ny + (size_t)y) * a.px + x;
    const int n = t.nst - 2;
    int i = 0;
    for (; i + 3 <= n; i += 3) {
        if (!t.plane_step(i, A, B, C, sh, out)) return false;
        if (!t.plane_step(i + 1, B, C, A, sh, out)) return false;
        if (!t.plane_step(i + 2, C, A, B, sh, out)) return false;
    }
    if (i < n) {
        if (!t.plane_step(i, A, B, C, sh, out)) return false;
        if (i + 1 < n && !t.plane_step(i + 1, B, C, A, sh, out)) return false;
    }
    jg = t.j0 + (uint32_t)t.nst;
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

template <typename T, int TY> constexpr int block_threads() { return 32 * TY / Lay<T>::RPW; }
// blocks per SM the register allocation must allow: at least 768 threads
template <typename T, int TY> constexpr int min_blocks()
{
    return block_threads<T, TY>() >= 768 ? 1 : 768 / block_threads<T, TY>();
}

template <typename T, int TY, int L, bool SR>
__global__ void __launch_bounds__(block_threads<T, TY>(), min_blocks<T, TY>()) k_step_tma(const __grid_constant__ StepArgs a,
                                                                        const __grid_constant__ CUtensorMap mP,
                                                                        const __grid_constant__ CUtensorMap mQ,
                                                                        const __grid_constant__ CUtensorMap mC, int *err)
{
    constexpr int D = L + 2;
    if (a.stop && *a.stop) return; // the stop rule fired at an earlier step (uniform over the block)
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + D * Stage<T, TY>::SB);
    init_bars<D>(bars);
    uint32_t jg = 0;
    step_tile<T, TY, L, SR>(a, &mP, &mQ, &mC, blockIdx.x, blockIdx.y, blockIdx.z, err, smem, bars, jg);
}

// Many simulations in one launch: the blocks walk the concatenated tile
// lists of all members (tiles of a member are consecutive, so neighbouring
// tiles run at the same time and share the halo rows in L2), either one
// tile per block or, persistent, a single wave of blocks striding over all.
template <typename T, int TY, int L, bool SR>
__global__ void __launch_bounds__(block_threads<T, TY>(), min_blocks<T, TY>()) k_step_tma_batch(const BatchMember *__restrict mem,
                                                                              uint32_t nmem, uint64_t ntiles,
                                                                              int parity, int *err)
{
    constexpr int D = L + 2;
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
        if (!step_tile<T, TY, L, SR>(b.step[parity], &b.mapP[parity], &b.mapQ[parity ^ 1], &b.mapC, bx, by, bz, err, smem,
                                 bars, jg))
            return;
    }
}

template <typename T, int TY, int L> constexpr size_t smem_bytes()
{
    return (size_t)(L + 2) * Stage<T, TY>::SB + (L + 2) * sizeof(uint64_t);
}

template <typename T, int TY, int L>
cudaError_t launch3(const StepArgs &a, const TmaMaps &m, int *err, cudaStream_t s)
{
    // stochastic rounding of the stores only exists for 16-bit storage
    auto kern = (sizeof(T) == 2 && a.sr) ? k_step_tma<T, TY, L, sizeof(T) == 2> : k_step_tma<T, TY, L, false>;
    constexpr size_t sm = smem_bytes<T, TY, L>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    if (a.ze <= a.zb) return cudaSuccess;
    const unsigned gx = (a.px + TX - 1) / TX;
    const unsigned gz = (unsigned)((a.ze - a.zb + a.zc - 1) / a.zc);
    kern<<<dim3(gx, (a.ny + TY - 1) / TY, gz), dim3(32, block_threads<T, TY>() / 32), sm, s>>>(a, *m.p, *m.q, *m.c,
                                                                                             err);
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
                          cudaStream_t s, bool mem_sr)
{
    auto kern = (sizeof(T) == 2 && mem_sr) ? k_step_tma_batch<T, TY, L, sizeof(T) == 2> : k_step_tma_batch<T, TY, L, false>;
    constexpr size_t sm = smem_bytes<T, TY, L>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, per = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, block_threads<T, TY>(), sm)) != cudaSuccess)
        return e;
    // persistent: one wave of blocks walks all tiles; otherwise one block per
    // tile and the hardware scheduler overlaps the blocks' prologues
    const uint64_t cap = persistent ? (uint64_t)nsm * (uint64_t)std::max(per, 1) : (uint64_t)INT32_MAX;
    const uint64_t grid = std::min<uint64_t>(ntiles, cap);
    kern<<<(unsigned)grid, dim3(32, block_threads<T, TY>() / 32), sm, s>>>(mem, nmem, ntiles, parity, err);
    return cudaGetLastError();
}

template <typename T, int TY>
cudaError_t launch_batch2(int depth, const BatchMember *mem, uint32_t nmem, uint64_t ntiles, int parity,
                          bool persistent, int *err, cudaStream_t s, bool sr)
{
    switch (depth) {
    case 1: return launch_batch3<T, TY, 1>(mem, nmem, ntiles, parity, persistent, err, s, sr);
    case 3: return launch_batch3<T, TY, 3>(mem, nmem, ntiles, parity, persistent, err, s, sr);
    default: return launch_batch3<T, TY, 2>(mem, nmem, ntiles, parity, persistent, err, s, sr);
    }
}

template <typename T>
cudaError_t launch_batch1(int rows, int depth, const BatchMember *mem, uint32_t nmem, uint64_t ntiles, int parity,
                          bool persistent, int *err, cudaStream_t s, bool sr)
{
    switch (rows) {
    case 4: return launch_batch2<T, 4>(depth, mem, nmem, ntiles, parity, persistent, err, s, sr);
    case 16: return launch_batch2<T, 16>(depth, mem, nmem, ntiles, parity, persistent, err, s, sr);
    default: return launch_batch2<T, 8>(depth, mem, nmem, ntiles, parity, persistent, err, s, sr);
    }
}

// ============================================================================
// Two steps in one pass (k_pair_tma)
// ============================================================================
// A block owns a tile of TX x TY voxels of (x, y), streamed along z as
// above, and computes p^{n+1} on the whole tile and p^{n+2} on its inner
// part: rows 1 .. TY-2 and the vectors 1 .. LPR-2 of each row (TX - 2V
// voxels).  Tiles overlap by one row and one vector on each side, so the
// inner parts cover the grid once; neighbouring tiles recompute the p^{n+1}
// of the overlap with the same operations, so every value agrees.  Along z
// a block computes p^{n+1} on the planes zs-1 .. z1 and p^{n+2} on
// zs .. z1-1.
//
// p^{n+1}(z) is computed from the staged planes exactly as k_step_tma does,
// rounded to the storage type, written to a two-plane ring in shared memory
// (for the y neighbours of the second step) and, on the inner part of the
// block's own planes, to p^{n+1} in global memory.  In the same iteration
// the block computes p^{n+2}(z-1): its centre and x neighbours are the
// thread's p^{n+1}(z-1) (registers, warp shuffles), its y neighbours come
// from the ring, its z neighbours are p^{n+1}(z-2) and p^{n+1}(z) in
// registers, and p^{n-1} of that step is the staged P(z-1).  Boundary,
// hard-source and border voxels keep the previous value in both steps, as
// in k_step_tma.
//
// Voxels whose p^{n+1} changes after the stencil (boundary voxels, by the
// boundary pass; hard and soft sources, by the post kernel) make the
// p^{n+2} of their air neighbours (and of a soft source itself) provisional:
// k_boundary_fix (kernels_step.cu) recomputes those from the final p^{n+1}
// in the launch of the second boundary pass, so two steps through this
// kernel give the results of two single steps bit for bit.  The fields are read once and written once per
// two steps: four buffers, p^n and p^{n-1} in, p^{n+1} and p^{n+2} out.
//
// The code box is TX + 16 bytes wide with its x origin rounded down to 16
// bytes (a TMA copy of 8-bit elements must start on a 16-byte boundary).
// A tile plane whose codes are all zero (a.tzmask, built per tiling by
// launch_pair_zero_masks) is not copied, as in k_step_tma.
template <typename T, int TY> struct PStage {
    static constexpr int CW = TX + 16;
    static constexpr uint32_t PB = Lay<T>::PW * (TY + 2) * sizeof(T);
    static constexpr uint32_t QB = TX * TY * sizeof(T);
    static constexpr uint32_t CB = CW * TY;
    static constexpr uint32_t PBa = (PB + 127u) & ~127u;
    static constexpr uint32_t QBa = (QB + 127u) & ~127u;
    static constexpr uint32_t CBa = (CB + 127u) & ~127u;
    static constexpr uint32_t SB = PBa + QBa + CBa;
    // one plane of p^{n+1} in the ring: TY + 2 rows (the first and the last
    // are read for tile rows 0 and TY-1, whose results are not kept)
    static constexpr uint32_t RB = ((TY + 2) * TX * sizeof(T) + 127u) & ~127u;
};

// a plain 16-byte store of V values (shared memory)
__device__ __forceinline__ void put_vec(float *p, const float (&r)[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(r[0], r[1], r[2], r[3]);
}
template <typename H> __device__ __forceinline__ void put_vec(H *p, const float (&r)[8])
{
    uint4 v;
    H *h = reinterpret_cast<H *>(&v);
#pragma unroll
    for (int k = 0; k < 8; ++k) h[k] = Io<H>::put(r[k]);
    *reinterpret_cast<uint4 *>(p) = v;
}

template <typename T, int TY, int L> struct PairTile {
    using S = PStage<T, TY>;
    using G = Lay<T>;
    static constexpr int D = L + 2, V = G::V;
    const StepArgs *a;
    unsigned char *smem;
    T *ring;
    uint64_t *bars;
    const CUtensorMap *mP, *mQ, *mC;
    int *err;
    T *zo, *wo; // this thread's voxel in plane 0 of p^{n+1} / p^{n+2}
    int xs, ys, zs, z1, xc, nst, sl, c0, t0, k0, r0;
    bool leader, inner;
    float2 c2dt2, inv_h2;
    size_t plane;
    uint64_t zmask; // bit j: the codes of stage j are all zero (not copied)

    __device__ __forceinline__ bool codes_zero(int j) const { return j < 64 && ((zmask >> j) & 1ull); }

    // stage j holds plane zs - 2 + j: P always, Q and the codes for the
    // planes zs-1 .. z1 (j = 1 .. nst-2)
    __device__ __forceinline__ void issue(int j) const
    {
        const int k = zs - 2 + j;
        unsigned char *st = smem + (uint32_t)(j % D) * S::SB;
        uint64_t *b = bars + (j % D);
        const bool full = j >= 1 && j <= nst - 2;
        const bool codes = full && !codes_zero(j);
        mbar_expect_tx(b, S::PB + (full ? S::QB : 0u) + (codes ? S::CB : 0u));
        tma_load_3d(st, mP, b, xs - G::PAD, ys - 1, k);
        if (full) tma_load_3d(st + S::PBa, mQ, b, xs, ys, k);
        if (codes) tma_load_3d(st + S::PBa + S::QBa, mC, b, xc, ys, k);
    }

    // Plane z = zs - 1 + i.  zm, cc: centres of P(z-1), P(z); zp receives
    // the centre of P(z+1).  um, uc: p^{n+1}(z-2), p^{n+1}(z-1); up
    // receives p^{n+1}(z).  cprev: the codes of plane z-1, replaced by those
    // of plane z.
    __device__ __forceinline__ bool plane_step(int i, const float (&zm)[V], const float (&cc)[V], float (&zp)[V],
                                               const float (&um)[V], const float (&uc)[V], float (&up)[V],
                                               Codes<V> &cprev, uint32_t &sh, T *&zout, T *&wout) const
    {
        using IO = Io<T>;
        constexpr int LPR = G::LPR, PW = G::PW;
        bool bad = false;
        if (leader) bad = !wait_stage(bars, (uint32_t)i + 2u, D, err);
        if (__syncthreads_or(bad)) return false;
        if (leader && i + D < nst) issue(i + D);
        const uint32_t sz = sh + 1u == (uint32_t)D ? 0u : sh + 1u;
        const int z = zs - 1 + i;

        // first step: p^{n+1}(z)
        const unsigned char *s0 = smem + sh * S::SB;
        const T *Ph = reinterpret_cast<const T *>(s0);
        {
            float ym[V], yp[V], qv[V];
            IO::ld(reinterpret_cast<const T *>(smem + sz * S::SB) + c0, zp);
            IO::ld(Ph + c0 - PW, ym);
            IO::ld(Ph + c0 + PW, yp);
            IO::ld(reinterpret_cast<const T *>(s0 + S::PBa) + t0, qv);
            Codes<V> code; // stage i + 1 holds plane z
            if (codes_zero(i + 1)) code.clear();
            else code.load(s0 + S::PBa + S::QBa + k0);
            float left = __shfl_up_sync(FULL, cc[V - 1], 1, LPR);
            float right = __shfl_down_sync(FULL, cc[0], 1, LPR);
            if (sl == 0) left = IO::ld1(Ph + c0 - 1);
            if (sl == LPR - 1) right = IO::ld1(Ph + c0 + V);
            tile_update<T>(code, cc, left, right, yp, ym, zp, zm, qv, c2dt2, inv_h2, a->c2dt2, a->inv_h2, up);
            T *rslot = ring + (uint32_t)(i & 1) * (S::RB / sizeof(T)) + r0;
            if constexpr (sizeof(T) == 2) {
                // rounded once: the packed vector goes to the ring and to
                // p^{n+1}, and its values feed the second step
                const uint4 pk = IO::pack(up);
                IO::unpack(pk, up);
                *reinterpret_cast<uint4 *>(rslot) = pk;
                if (inner && z >= zs && z < z1) IO::st_packed(zout, pk);
            } else {
                put_vec(rslot, up);
                if (inner && z >= zs && z < z1) IO::st(zout, up);
            }
            zout += plane;
            // second step: p^{n+2}(z-1), from the ring plane written in the
            // previous iteration (visible since this iteration's barrier).
            // Computed in every iteration, without a branch, so that the
            // compiler can interleave it with the first step; kept from
            // i = 2 on (the first two planes are the halo below the block).
            {
                const T *rm = ring + (uint32_t)((i - 1) & 1) * (S::RB / sizeof(T)) + r0;
                float ym2[V], yp2[V], r2[V];
                IO::ld(rm - TX, ym2);
                IO::ld(rm + TX, yp2);
                const float left2 = __shfl_up_sync(FULL, uc[V - 1], 1, LPR);
                const float right2 = __shfl_down_sync(FULL, uc[0], 1, LPR);
                tile_update<T>(cprev, uc, left2, right2, yp2, ym2, up, um, zm, c2dt2, inv_h2, a->c2dt2, a->inv_h2,
                               r2);
                if (inner && i >= 2) IO::st(wout, r2);
                if (i >= 2) wout += plane;
            }
            cprev = code;
        }
        sh = sz;
        return true;
    }
};

// blocks per SM the register allocation must allow: two FP32 blocks of 512
// threads (64 registers, no spills); the 16-bit kernels keep their registers
template <typename T, int TY> constexpr int pair_min_blocks()
{
    return sizeof(T) == 4 && block_threads<T, TY>() <= 512 ? 2 : 1;
}

template <typename T, int TY, int L>
__global__ void __launch_bounds__(block_threads<T, TY>(), (pair_min_blocks<T, TY>())) k_pair_tma(const __grid_constant__ StepArgs a,
                                                                        const __grid_constant__ CUtensorMap mP,
                                                                        const __grid_constant__ CUtensorMap mQ,
                                                                        const __grid_constant__ CUtensorMap mC,
                                                                        void *zout, void *wout, int *err)
{
    using G = Lay<T>;
    using S = PStage<T, TY>;
    using IO = Io<T>;
    constexpr int V = G::V, LPR = G::LPR, PW = G::PW, PAD = G::PAD, D = L + 2;
    constexpr int IX = TX - 2 * V, IY = TY - 2;
    if (a.stop && *a.stop) return; // the stop rule fired at an earlier step (uniform over the block)
    extern __shared__ __align__(128) unsigned char smem[];
    PairTile<T, TY, L> t;
    t.a = &a;
    t.smem = smem;
    t.ring = reinterpret_cast<T *>(smem + D * S::SB);
    t.bars = reinterpret_cast<uint64_t *>(smem + D * S::SB + 2 * S::RB);
    t.mP = &mP;
    t.mQ = &mQ;
    t.mC = &mC;
    t.err = err;
    const int lane = threadIdx.x, tid = threadIdx.y * 32 + lane;
    for (uint32_t k = tid; k < 2 * S::RB / 16; k += blockDim.x * blockDim.y)
        reinterpret_cast<uint4 *>(t.ring)[k] = make_uint4(0u, 0u, 0u, 0u);
    init_bars<D>(t.bars);
    t.zs = 1 + (int)blockIdx.z * a.zc;
    t.z1 = min(t.zs + a.zc, (int)a.nz - 1);
    if (t.zs >= t.z1) return; // uniform over the block
    t.nst = t.z1 - t.zs + 4;  // P planes zs-2 .. z1+1
    t.xs = (int)blockIdx.x * IX - V;
    t.ys = (int)blockIdx.y * IY - 1;
    t.xc = t.xs & ~15; // rounded down to 16 bytes of codes (two's complement: also below zero)
    const int row = threadIdx.y * G::RPW + lane / LPR;
    t.sl = lane % LPR;
    const int x = t.xs + t.sl * V, y = t.ys + row;
    t.inner = t.sl >= 1 && t.sl <= LPR - 2 && row >= 1 && row <= TY - 2 && x < (int)a.px && y < (int)a.ny;
    t.leader = tid == 0;
    t.c0 = (row + 1) * PW + PAD + t.sl * V;
    t.t0 = row * TX + t.sl * V;
    t.k0 = row * S::CW + (t.xs - t.xc) + t.sl * V;
    t.r0 = (row + 1) * TX + t.sl * V;
    t.c2dt2 = make_float2(a.c2dt2, a.c2dt2);
    t.inv_h2 = make_float2(a.inv_h2, a.inv_h2);
    t.plane = (size_t)a.px * a.ny;
    t.zmask = a.tzmask ? __ldg(a.tzmask + ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x)
                       : 0ull;
    const size_t off = t.inner ? (size_t)y * a.px + (size_t)x : 0;
    t.zo = static_cast<T *>(zout) + off;
    t.wo = static_cast<T *>(wout) + off;
    T *zrun = t.zo + (size_t)(t.zs - 1) * t.plane; // p^{n+1} of the plane of the current iteration
    T *wrun = t.wo + (size_t)t.zs * t.plane;       // p^{n+2} of the plane the second step writes next

    if (t.leader)
        for (int j = 0; j < D && j < t.nst; ++j) t.issue(j);

    float A[V], B[V], C[V], X0[V], X1[V], X2[V];
#pragma unroll
    for (int k = 0; k < V; ++k) X0[k] = X1[k] = X2[k] = 0.f;
    {
        bool bad = false;
        if (t.leader) bad = !wait_stage(t.bars, 0u, D, err) || !wait_stage(t.bars, 1u, D, err);
        if (__syncthreads_or(bad)) return;
        IO::ld(reinterpret_cast<const T *>(smem) + t.c0, A);                        // P(zs-2)
        IO::ld(reinterpret_cast<const T *>(smem + (1u % D) * S::SB) + t.c0, B);     // P(zs-1)
    }
    uint32_t sh = 1u % D;
    Codes<V> cprev;
    cprev.clear();
    // i = 0 .. n-1 computes p^{n+1} of plane zs-1+i; the p^{n+1} centres
    // rotate through X0..X2 with the P centres A..C, three planes per turn
    const int n = t.nst - 2;
    int i = 0;
    for (; i + 3 <= n; i += 3) {
        if (!t.plane_step(i, A, B, C, X1, X2, X0, cprev, sh, zrun, wrun)) return;
        if (!t.plane_step(i + 1, B, C, A, X2, X0, X1, cprev, sh, zrun, wrun)) return;
        if (!t.plane_step(i + 2, C, A, B, X0, X1, X2, cprev, sh, zrun, wrun)) return;
    }
    if (i < n) {
        if (!t.plane_step(i, A, B, C, X1, X2, X0, cprev, sh, zrun, wrun)) return;
        if (i + 1 < n && !t.plane_step(i + 1, B, C, A, X2, X0, X1, cprev, sh, zrun, wrun)) return;
    }
}

template <typename T, int TY, int L> constexpr size_t pair_smem_bytes()
{
    return (size_t)(L + 2) * PStage<T, TY>::SB + 2 * PStage<T, TY>::RB + (L + 2) * sizeof(uint64_t);
}

template <typename T, int TY, int L>
cudaError_t pair3(const StepArgs &a, const TmaMaps &m, void *zout, void *wout, int *err, cudaStream_t s)
{
    auto kern = k_pair_tma<T, TY, L>;
    constexpr size_t sm = pair_smem_bytes<T, TY, L>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    constexpr int IX = TX - 2 * Lay<T>::V, IY = TY - 2;
    const unsigned gx = (a.px + IX - 1) / IX, gy = (a.ny + IY - 1) / IY;
    const unsigned gz = (a.nz - 2 + a.zc - 1) / a.zc;
    kern<<<dim3(gx, gy, gz), dim3(32, block_threads<T, TY>() / 32), sm, s>>>(a, *m.p, *m.q, *m.c, zout, wout, err);
    return cudaGetLastError();
}

// planes in flight per tile height: as many as two FP32 blocks per SM
// leave room for (12 rows: 4, 14 rows: 3, 16 rows: 2); the 32-row tile fills
// an SM alone and keeps 2
template <typename T>
cudaError_t pair1(int rows, const StepArgs &a, const TmaMaps &m, void *zout, void *wout, int *err, cudaStream_t s)
{
    switch (rows) {
    case 12: return pair3<T, 12, 4>(a, m, zout, wout, err, s);
    case 14: return pair3<T, 14, 3>(a, m, zout, wout, err, s);
    case 32: return pair3<T, 32, 2>(a, m, zout, wout, err, s);
    default: return pair3<T, 16, 2>(a, m, zout, wout, err, s);
    }
}

} // namespace

cudaError_t launch_step_tma_batch(int storage, int tile_rows, int depth, const BatchMember *mem, uint32_t nmem,
                                  uint64_t ntiles, int parity, bool persistent, int *err, cudaStream_t s, bool sr)
{
    if (ntiles == 0) return cudaSuccess;
    switch (storage) {
    case VIRS_STORAGE_F16:
        return launch_batch1<__half>(tile_rows, depth, mem, nmem, ntiles, parity, persistent, err, s, sr);
    case VIRS_STORAGE_BF16:
        return launch_batch1<__nv_bfloat16>(tile_rows, depth, mem, nmem, ntiles, parity, persistent, err, s, sr);
    default: return launch_batch1<float>(tile_rows, depth, mem, nmem, ntiles, parity, persistent, err, s, false);
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

int pair_tile_x(int storage) { return TX - 2 * (storage == VIRS_STORAGE_F32 ? 4 : 8); }
int pair_code_box() { return TX + 16; }

cudaError_t launch_pair_tma(int storage, int tile_rows, const StepArgs &a0, const TmaMaps &m, void *zout, void *wout,
                            int *err, cudaStream_t s)
{
    if (a0.nz < 3 || a0.ny < 3 || a0.nx < 3) return cudaSuccess;
    StepArgs a = a0;
    if (a.zc <= 0) a.zc = (int)a.nz - 2;
    switch (storage) {
    case VIRS_STORAGE_F16: return pair1<__half>(tile_rows, a, m, zout, wout, err, s);
    case VIRS_STORAGE_BF16: return pair1<__nv_bfloat16>(tile_rows, a, m, zout, wout, err, s);
    default: return pair1<float>(tile_rows, a, m, zout, wout, err, s);
    }
}


} // namespace virs
