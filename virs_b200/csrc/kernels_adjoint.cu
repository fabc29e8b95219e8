// Reverse-mode (adjoint) kernels: gradients of a receiver loss with respect
// to the boundary filter coefficients and the source signals.
//
// One forward step maps (p, q, S) -> (p+, p, S+), linear in the fields and
// the filter states.  With T the adjoint of p^{n+1} and RR the negated
// adjoint carried by p^n through its role as q of the next step, one
// reverse step n is
//   k_adj_inject     T[rcv] += dL/dIR_n ; dL/dsig_n = T[src]
//   k_adj_boundary   at boundary voxels the correction and the biquad cascade
//                    run transposed: F = T (reference form) or T/(1+a)
//                    (centered form), the cascade's state adjoints and the
//                    coefficient gradients (FP64), dbar = d(loss)/d(p - q)
//   stencil          T' = A F - RR into RR's buffer: the forward stencil
//                    kernel itself, since A (2 + lambda^2 * Laplacian with
//                    mirrored walls and zero fixed voxels) is symmetric on
//                    the updated voxels; hard-source voxels are given 0
//   k_adj_fix        boundary voxels: T'_b = A F_b - RR_b + dbar_b (from the
//                    stencil's record) and RR'_b = F_b + dbar_b - cq_b
// and the buffers swap.  The forward values the cascade needs (p - q and
// the states before step n) come from a recomputation of the segment from
// the last checkpoint.
#include "step_common.cuh"

namespace virs {
namespace {

using namespace step;

__global__ void k_adj_inject(float *T, const uint8_t *__restrict code, const uint64_t *__restrict rcv, uint32_t nrcv,
                             const float *__restrict dl, uint64_t dl_stride, uint64_t n, const uint64_t *__restrict src,
                             uint32_t nsrc, float *__restrict gsig, uint64_t gs_stride)
{
    for (uint32_t r = threadIdx.x; r < nrcv; r += blockDim.x) {
        // receivers read the new field; a receiver on a voxel that is not
        // updated (wall, hard source, border) reads a constant
        const uint64_t i = rcv[r];
        if (code[i] < CODE_HARD) atomicAdd(T + i, dl[(uint64_t)r * dl_stride + n]);
    }
    __syncthreads();
    for (uint32_t s = threadIdx.x; s < nsrc; s += blockDim.x) gsig[(uint64_t)s * gs_stride + n] = T[src[s]];
}

struct AdjArgs {
    float *T;                  // adjoint field (p role)
    const uint32_t *bidx;
    const uint8_t *bmat;
    const float *bw;
    const float *coef;         // [M][S][5]
    const float4 *rec;         // forward records of this step {free, p, q, 0}
    const float *fst;          // forward states before this step (the cascade's layout, state_index)
    float *ast;                // state adjoints, four per section [S][4][nb]
    float *dbar, *cq;          // per slot
    double *grad;              // [M][S][5]
    uint64_t nb;
    uint32_t nx, ny, px, nsec, ncoef;
    int form;
    double K, mix_y, mix_d, gain;
};

constexpr int AB = 256;

// The shuffle schedule of peer_sum for one lane, worked out once and used
// for every sum of a slot: in round r the lane takes the value of lane
// src[r] and adds it when bit r of `use` is set; `rounds` (at most five,
// for a group of 32) is the same on every lane.
struct PeerPlan {
    int src[5];
    unsigned use;
    int rounds;
};

__device__ __forceinline__ PeerPlan peer_plan(unsigned peers)
{
    PeerPlan p;
    p.use = 0u;
    p.rounds = 0;
    const int lane = (int)(threadIdx.x & 31u);
    unsigned rank = __popc(peers & ((1u << lane) - 1u));
    peers &= 0xfffffffeu << lane;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        p.src[r] = lane;
        if (__any_sync(0xffffffffu, peers != 0u)) {
            const int next = __ffs(peers);
            if (next > 0) {
                p.src[r] = next - 1;
                p.use |= 1u << r;
            }
            peers &= __ballot_sync(0xffffffffu, (rank & 1u) == 0u);
            rank >>= 1;
            p.rounds = r + 1;
        }
    }
    return p;
}

// peer_sum with a schedule from peer_plan
__device__ __forceinline__ double plan_sum(const PeerPlan &p, double v)
{
#pragma unroll
    for (int r = 0; r < 5; ++r)
        if (r < p.rounds) {
            const double u = __shfl_sync(0xffffffffu, v, p.src[r]);
            if ((p.use >> r) & 1u) v += u;
        }
    return v;
}

// The sum of v over the lanes of a full warp that share this lane's key
// (peers = __match_any_sync of the key), complete at the group's lowest
// lane: a tree over each group's ranks, every lane taking part in every
// shuffle.  Lanes of a mixed warp (boundary slots of two or more
// materials) then make one shared-memory add per group instead of one
// each.
__device__ __forceinline__ double peer_sum(unsigned peers, double v)
{
    const unsigned lane = threadIdx.x & 31u;
    unsigned rank = __popc(peers & ((1u << lane) - 1u));
    peers &= 0xfffffffeu << lane; // the peers above this lane
    while (__any_sync(0xffffffffu, peers != 0u)) {
        const int next = __ffs(peers);
        const double u = __shfl_sync(0xffffffffu, v, next > 0 ? next - 1 : 0);
        if (next > 0) v += u;
        peers &= __ballot_sync(0xffffffffu, (rank & 1u) == 0u);
        rank >>= 1;
    }
    return v;
}

__global__ void __launch_bounds__(AB) k_adj_boundary(const AdjArgs a)
{
    extern __shared__ double gsm[]; // block partial sums of the coefficient gradients
    for (uint32_t k = threadIdx.x; k < a.ncoef; k += AB) gsm[k] = 0.0;
    __syncthreads();
    const uint64_t b = (uint64_t)blockIdx.x * AB + threadIdx.x;
    if (b < a.nb) {
        const uint32_t ref = a.bidx[b];
        const uint32_t x = ref % a.nx, t = ref / a.nx, y = t % a.ny, z = t / a.ny;
        const size_t i = ((size_t)z * a.ny + y) * a.px + x;
        const float f = a.T[i];
        const double w = (double)a.bw[b];
        const double kgw = a.K * a.gain * w;
        double fr, ybar, db = 0.0, cqv = 0.0;
        if (a.form == VIRS_BOUNDARY_REFERENCE) {
            fr = f;
            ybar = -kgw * a.mix_y * f;
            db = -kgw * a.mix_d * f;
        } else {
            const double ac = kgw * a.mix_d * 0.5;
            fr = f / (1.0 + ac);
            ybar = -kgw * a.mix_y * fr;
            cqv = ac * fr;
        }
        // forward inputs of every section at this step
        const uint32_t S = a.nsec, m = a.bmat[b];
        const float *kc = a.coef + (uint64_t)m * S * 5;
        const float4 rec = a.rec[b];
        float xin[16];
        float in = __fsub_rn(rec.y, rec.z);
        for (uint32_t q = 0; q < S; ++q) {
            const float *kq = kc + 5 * q;
            const float s0 = a.fst[state_index(2 * q + 0, b, a.nb)], s1 = a.fst[state_index(2 * q + 1, b, a.nb)];
            const float s2 = a.fst[state_index(2 * q + 2, b, a.nb)], s3 = a.fst[state_index(2 * q + 3, b, a.nb)];
            xin[q] = in;
            float yv = __fmaf_rn(kq[0], in, __fmul_rn(kq[1], s0));
            yv = __fmaf_rn(kq[2], s1, yv);
            yv = __fmaf_rn(-kq[3], s2, yv);
            in = __fmaf_rn(-kq[4], s3, yv);
        }
        // every lane of this warp holds a slot of one material (the loops
        // over the sections are uniform: S is the same for every slot)
        // full warps sum over the lanes of each material first
        const bool full = __activemask() == 0xffffffffu;
        const unsigned peers = full ? __match_any_sync(0xffffffffu, m) : 0u;
        const bool lead = full && (int)(threadIdx.x & 31u) == __ffs(peers) - 1;
        double yb = ybar;
        for (int q = (int)S - 1; q >= 0; --q) {
            const float *kq = kc + 5 * q;
            float *aq = a.ast + b;
            const uint64_t o0 = (uint64_t)(4 * q + 0) * a.nb, o1 = (uint64_t)(4 * q + 1) * a.nb;
            const uint64_t o2 = (uint64_t)(4 * q + 2) * a.nb, o3 = (uint64_t)(4 * q + 3) * a.nb;
            const double yt = yb + (double)aq[o2];
            const double s0 = a.fst[state_index(2 * q, b, a.nb)], s1 = a.fst[state_index(2 * q + 1, b, a.nb)],
                         s2 = a.fst[state_index(2 * q + 2, b, a.nb)], s3 = a.fst[state_index(2 * q + 3, b, a.nb)];
            double *g = gsm + (uint64_t)(m * S + q) * 5;
            const double gv[5] = {yt * (double)xin[q], yt * s0, yt * s1, -yt * s2, -yt * s3};
            if (full) {
#pragma unroll
                for (int j = 0; j < 5; ++j) {
                    const double v = peer_sum(peers, gv[j]);
                    if (lead) atomicAdd(g + j, v);
                }
            } else {
#pragma unroll
                for (int j = 0; j < 5; ++j) atomicAdd(g + j, gv[j]);
            }
            const double xbar = (double)kq[0] * yt + (double)aq[o0];
            const double x1 = (double)kq[1] * yt + (double)aq[o1];
            const double x2 = (double)kq[2] * yt;
            const double y1 = -(double)kq[3] * yt + (double)aq[o3];
            const double y2 = -(double)kq[4] * yt;
            aq[o0] = (float)x1;
            aq[o1] = (float)x2;
            aq[o2] = (float)y1;
            aq[o3] = (float)y2;
            yb = xbar;
        }
        db += yb;
        a.T[i] = (float)fr;
        a.dbar[b] = (float)db;
        a.cq[b] = (float)cqv;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < a.ncoef; k += AB)
        if (gsm[k] != 0.0) atomicAdd(a.grad + k, gsm[k]);
}

constexpr int ABS = 128; // threads per block of k_adj_boundary_s: a few slots per SM at small sizes still fill it

// The same for cascades of up to MAXS sections, unrolled: the forward
// section inputs and the filter states stay in registers (the states are
// read once, as the 16-byte groups of the cascade's layout).
template <int MAXS> __global__ void __launch_bounds__(ABS) k_adj_boundary_s(const AdjArgs a)
{
    constexpr int NG = (2 * (MAXS + 1) + 3) / 4;
    extern __shared__ double gsm[]; // block partial sums of the coefficient gradients
    for (uint32_t k = threadIdx.x; k < a.ncoef; k += ABS) gsm[k] = 0.0;
    __syncthreads();
    const uint64_t b = (uint64_t)blockIdx.x * ABS + threadIdx.x;
    if (b < a.nb) {
        const uint32_t ref = a.bidx[b];
        const uint32_t S = a.nsec, m = a.bmat[b];
        const float4 rec = a.rec[b];
        const double w = (double)a.bw[b];
        float h[4 * NG];
        const float4 *st = reinterpret_cast<const float4 *>(a.fst) + b;
        const uint32_t ng = (2u * (S + 1u) + 3u) / 4u;
#pragma unroll
        for (int g = 0; g < NG; ++g)
            if ((uint32_t)g < ng) {
                const float4 v = st[(uint64_t)g * a.nb];
                h[4 * g] = v.x;
                h[4 * g + 1] = v.y;
                h[4 * g + 2] = v.z;
                h[4 * g + 3] = v.w;
            }
        const uint32_t x = ref % a.nx, t = ref / a.nx, y = t % a.ny, z = t / a.ny;
        const size_t i = ((size_t)z * a.ny + y) * a.px + x;
        const float f = a.T[i];
        const double kgw = a.K * a.gain * w;
        double fr, ybar, db = 0.0, cqv = 0.0;
        if (a.form == VIRS_BOUNDARY_REFERENCE) {
            fr = f;
            ybar = -kgw * a.mix_y * f;
            db = -kgw * a.mix_d * f;
        } else {
            const double ac = kgw * a.mix_d * 0.5;
            fr = f / (1.0 + ac);
            ybar = -kgw * a.mix_y * fr;
            cqv = ac * fr;
        }
        // forward inputs of every section at this step
        const float *kc = a.coef + (uint64_t)m * S * 5;
        float xin[MAXS];
        float in = __fsub_rn(rec.y, rec.z);
#pragma unroll
        for (int q = 0; q < MAXS; ++q)
            if (q < (int)S) {
                const float *kq = kc + 5 * q;
                xin[q] = in;
                float yv = __fmaf_rn(kq[0], in, __fmul_rn(kq[1], h[2 * q]));
                yv = __fmaf_rn(kq[2], h[2 * q + 1], yv);
                yv = __fmaf_rn(-kq[3], h[2 * q + 2], yv);
                in = __fmaf_rn(-kq[4], h[2 * q + 3], yv);
            }
        const bool full = __activemask() == 0xffffffffu;
        const unsigned peers = full ? __match_any_sync(0xffffffffu, m) : 0u;
        const bool lead = full && (int)(threadIdx.x & 31u) == __ffs(peers) - 1;
        const PeerPlan plan = full ? peer_plan(peers) : PeerPlan{};
        double yb = ybar;
#pragma unroll
        for (int q = MAXS - 1; q >= 0; --q)
            if (q < (int)S) {
                const float *kq = kc + 5 * q;
                float *aq = a.ast + b;
                const uint64_t o0 = (uint64_t)(4 * q + 0) * a.nb, o1 = (uint64_t)(4 * q + 1) * a.nb;
                const uint64_t o2 = (uint64_t)(4 * q + 2) * a.nb, o3 = (uint64_t)(4 * q + 3) * a.nb;
                const double yt = yb + (double)aq[o2];
                double *g = gsm + (uint64_t)(m * S + q) * 5;
                const double gv[5] = {yt * (double)xin[q], yt * (double)h[2 * q], yt * (double)h[2 * q + 1],
                                      -yt * (double)h[2 * q + 2], -yt * (double)h[2 * q + 3]};
                if (full) {
#pragma unroll
                    for (int j = 0; j < 5; ++j) {
                        const double v = plan_sum(plan, gv[j]);
                        if (lead) atomicAdd(g + j, v);
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 5; ++j) atomicAdd(g + j, gv[j]);
                }
                const double xbar = (double)kq[0] * yt + (double)aq[o0];
                const double x1 = (double)kq[1] * yt + (double)aq[o1];
                const double x2 = (double)kq[2] * yt;
                const double y1 = -(double)kq[3] * yt + (double)aq[o3];
                const double y2 = -(double)kq[4] * yt;
                aq[o0] = (float)x1;
                aq[o1] = (float)x2;
                aq[o2] = (float)y1;
                aq[o3] = (float)y2;
                yb = xbar;
            }
        db += yb;
        a.T[i] = (float)fr;
        a.dbar[b] = (float)db;
        a.cq[b] = (float)cqv;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < a.ncoef; k += ABS)
        if (gsm[k] != 0.0) atomicAdd(a.grad + k, gsm[k]);
}

// boundary voxels after the stencil: T' (in RR's buffer) and the next RR
// (in T's buffer)
__global__ void k_adj_fix(float *Tn, float *Tb, const uint32_t *__restrict bidx, const float4 *__restrict rec,
                          const float *__restrict dbar, const float *__restrict cq, uint64_t nb, uint32_t nx,
                          uint32_t ny, uint32_t px)
{
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint32_t ref = bidx[b];
    const uint32_t x = ref % nx, t = ref / nx, y = t % ny, z = t / ny;
    const size_t i = ((size_t)z * ny + y) * px + x;
    Tn[i] = rec[b].x + dbar[b];
    Tb[i] = Tb[i] + dbar[b] - cq[b];
}

} // namespace

cudaError_t launch_adj_inject(float *T, const uint8_t *code, const uint64_t *rcv, uint32_t nrcv, const float *dl,
                              uint64_t dl_stride, uint64_t n, const uint64_t *src, uint32_t nsrc, float *gsig,
                              uint64_t gs_stride, cudaStream_t s)
{
    k_adj_inject<<<1, 256, 0, s>>>(T, code, rcv, nrcv, dl, dl_stride, n, src, nsrc, gsig, gs_stride);
    return cudaGetLastError();
}

cudaError_t launch_adj_boundary(float *T, const uint32_t *bidx, const uint8_t *bmat, const float *bw, const float *coef,
                                const float4 *rec, const float *fst, float *ast, float *dbar, float *cq, double *grad,
                                uint64_t nb, uint32_t nx, uint32_t ny, uint32_t px, uint32_t nsec, uint32_t nmat,
                                int form, double K, double mix_y, double mix_d, double gain, cudaStream_t s)
{
    if (nb == 0) return cudaSuccess;
    AdjArgs a{T, bidx, bmat, bw, coef, rec, fst, ast, dbar, cq, grad, nb, nx, ny, px, nsec, nmat * nsec * 5, form,
              K, mix_y, mix_d, gain};
    const size_t sm = (size_t)a.ncoef * sizeof(double);
    const unsigned gs = (unsigned)((nb + ABS - 1) / ABS);
    if (nsec <= 1) k_adj_boundary_s<1><<<gs, ABS, sm, s>>>(a);
    else if (nsec == 2) k_adj_boundary_s<2><<<gs, ABS, sm, s>>>(a);
    else if (nsec <= 4) k_adj_boundary_s<4><<<gs, ABS, sm, s>>>(a);
    else k_adj_boundary<<<(unsigned)((nb + AB - 1) / AB), AB, sm, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adj_fix(float *Tn, float *Tb, const uint32_t *bidx, const float4 *rec, const float *dbar,
                           const float *cq, uint64_t nb, uint32_t nx, uint32_t ny, uint32_t px, cudaStream_t s)
{
    if (nb == 0) return cudaSuccess;
    k_adj_fix<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(Tn, Tb, bidx, rec, dbar, cq, nb, nx, ny, px);
    return cudaGetLastError();
}

namespace {
__global__ void k_zero_at(float *f, const uint32_t *__restrict pos, uint32_t n)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) f[pos[k]] = 0.f;
}
} // namespace

// the adjoint at the hard-source voxels is 0 (their forward value does not
// depend on the field); the stencil leaves them alone
cudaError_t launch_zero_at(float *f, const uint32_t *pos, uint32_t n, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_zero_at<<<(n + 255) / 256, 256, 0, s>>>(f, pos, n);
    return cudaGetLastError();
}

namespace {
__global__ void k_set_u32(uint32_t *p, uint32_t v) { *p = v; }
} // namespace

// one device word set in stream order (no host staging buffer)
cudaError_t launch_set_u32(uint32_t *p, uint32_t v, cudaStream_t s)
{
    k_set_u32<<<1, 1, 0, s>>>(p, v);
    return cudaGetLastError();
}

} // namespace virs
