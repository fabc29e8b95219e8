// Device helpers shared by the stencil kernels: storage types, the
// leapfrog update and the boundary correction, with the arithmetic order of
// the reference build written out (see kernels_step.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "internal.hpp"

namespace virs {
namespace step {
namespace {

constexpr unsigned FULL = 0xffffffffu;

// ---- storage types ------------------------------------------------------------

template <typename T> struct Io;

template <> struct Io<float> {
    static constexpr int VEC = 4;
    __device__ static void ld(const float *p, float (&r)[VEC])
    {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
    }
    __device__ static void ld_stream(const float *p, float (&r)[VEC])
    {
        const float4 v = __ldcs(reinterpret_cast<const float4 *>(p));
        r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
    }
    __device__ static void st(float *p, const float (&r)[VEC])
    {
        __stcs(reinterpret_cast<float4 *>(p), make_float4(r[0], r[1], r[2], r[3]));
    }
    __device__ static float ld1(const float *p) { return *p; }
    __device__ static float get(float v) { return v; }
    __device__ static float put(float v) { return v; }
};

template <> struct Io<__half> {
    static constexpr int VEC = 8;
    __device__ static void unpack(const uint4 v, float (&r)[VEC])
    {
        const __half2 *h = reinterpret_cast<const __half2 *>(&v);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 f = __half22float2(h[i]);
            r[2 * i] = f.x;
            r[2 * i + 1] = f.y;
        }
    }
    __device__ static void ld(const __half *p, float (&r)[VEC]) { unpack(*reinterpret_cast<const uint4 *>(p), r); }
    __device__ static void ld_stream(const __half *p, float (&r)[VEC]) { unpack(__ldcs(reinterpret_cast<const uint4 *>(p)), r); }
    __device__ static void st(__half *p, const float (&r)[VEC])
    {
        uint4 v;
        __half2 *h = reinterpret_cast<__half2 *>(&v);
#pragma unroll
        for (int i = 0; i < 4; ++i) h[i] = __floats2half2_rn(r[2 * i], r[2 * i + 1]);
        __stcs(reinterpret_cast<uint4 *>(p), v);
    }
    // V values rounded to FP16 in one 16-byte vector, and a streaming store of one
    __device__ static uint4 pack(const float (&r)[VEC])
    {
        uint4 v;
        __half2 *h = reinterpret_cast<__half2 *>(&v);
#pragma unroll
        for (int i = 0; i < 4; ++i) h[i] = __floats2half2_rn(r[2 * i], r[2 * i + 1]);
        return v;
    }
    __device__ static void st_packed(__half *p, uint4 v) { __stcs(reinterpret_cast<uint4 *>(p), v); }
    __device__ static float ld1(const __half *p) { return __half2float(*p); }
    __device__ static float get(__half v) { return __half2float(v); }
    __device__ static __half put(float v) { return __float2half_rn(v); }
};

template <> struct Io<__nv_bfloat16> {
    static constexpr int VEC = 8;
    __device__ static void unpack(const uint4 v, float (&r)[VEC])
    {
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 f = __bfloat1622float2(h[i]);
            r[2 * i] = f.x;
            r[2 * i + 1] = f.y;
        }
    }
    __device__ static void ld(const __nv_bfloat16 *p, float (&r)[VEC]) { unpack(*reinterpret_cast<const uint4 *>(p), r); }
    __device__ static void ld_stream(const __nv_bfloat16 *p, float (&r)[VEC])
    {
        unpack(__ldcs(reinterpret_cast<const uint4 *>(p)), r);
    }
    __device__ static void st(__nv_bfloat16 *p, const float (&r)[VEC])
    {
        uint4 v;
        __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&v);
#pragma unroll
        for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(r[2 * i], r[2 * i + 1]);
        __stcs(reinterpret_cast<uint4 *>(p), v);
    }
    __device__ static uint4 pack(const float (&r)[VEC])
    {
        uint4 v;
        __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&v);
#pragma unroll
        for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(r[2 * i], r[2 * i + 1]);
        return v;
    }
    __device__ static void st_packed(__nv_bfloat16 *p, uint4 v) { __stcs(reinterpret_cast<uint4 *>(p), v); }
    __device__ static float ld1(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
    __device__ static float get(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ static __nv_bfloat16 put(float v) { return __float2bfloat16_rn(v); }
};

// ---- stochastic rounding of the 16-bit stores (opt-in) -----------------------
//
// With VIRS_ROUND_STOCHASTIC a value stored as FP16 / BF16 is rounded up in
// magnitude with a probability equal to the fraction it lies between its two
// neighbours, instead of to the nearest: 16 random bits are added below the
// kept bits of the FP32 pattern, which is then truncated.  The bits are a
// pure function of (voxel, step, phase), so runs are reproducible and every
// kernel variant rounds a voxel alike:
//   s    = mix32(2 * step + phase + SR_SEED)      phase 0: the step's store of
//                                                 p^{n+1} (stencil, boundary pass,
//                                                 hard source); 1: soft sources
//   w    = mix32((pos + base) / 2 ^ s)            pos: padded device index;
//                                                 base: a slab's offset in the
//                                                 whole grid (0 otherwise)
//   bits = low 16 of w for an even position, high 16 for an odd one
// mix32 is Chris Wellons' "lowbias32" integer hash (hash-prospector, public
// domain).  Values that round to themselves (exact ones: walls, kept
// p^{n-1}) are unchanged; FP16 values below 2^-14 or from 65504 up in
// magnitude, and non-finite values, round to nearest.
constexpr uint32_t SR_SEED = 0x9e3779b9u;

__device__ __forceinline__ uint32_t mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// the per-launch part of the key
__device__ __forceinline__ uint32_t sr_step_key(uint32_t step, uint32_t phase)
{
    return mix32(2u * step + phase + SR_SEED);
}

// the random word of the voxel pair holding padded position pos
__device__ __forceinline__ uint32_t sr_word(uint64_t pos, uint64_t base, uint32_t key)
{
    return mix32((uint32_t)((pos + base) >> 1) ^ key);
}

__device__ __forceinline__ uint32_t sr_bits(uint64_t pos, uint64_t base, uint32_t key)
{
    const uint32_t w = sr_word(pos, base, key);
    return ((pos + base) & 1u) ? (w >> 16) : (w & 0xffffu);
}

// FP32 pattern rounded stochastically to the kept bits of T (truncated,
// exactly representable in T), or to nearest where stated above
__device__ __forceinline__ __nv_bfloat16 sr_bf16(float f, uint32_t r16)
{
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7fffffffu) < 0x7f7f0000u) {
        u = (u + r16) & 0xffff0000u;
        return __ushort_as_bfloat16((unsigned short)(u >> 16));
    }
    return __float2bfloat16_rn(f);
}

__device__ __forceinline__ __half sr_f16(float f, uint32_t r16)
{
    const uint32_t u = __float_as_uint(f), a = u & 0x7fffffffu;
    if (a >= 0x38800000u && a < 0x477fe000u) return __float2half_rn(__uint_as_float((u + (r16 & 0x1fffu)) & ~0x1fffu));
    return __float2half_rn(f);
}

template <typename T> struct Sr;
template <> struct Sr<float> {
    __device__ static float put(float f, uint32_t) { return f; }
};
template <> struct Sr<__nv_bfloat16> {
    __device__ static __nv_bfloat16 put(float f, uint32_t r16) { return sr_bf16(f, r16); }
};
template <> struct Sr<__half> {
    __device__ static __half put(float f, uint32_t r16) { return sr_f16(f, r16); }
};

// a store of one value: to nearest, or stochastic with `key` (sr != 0)
template <typename T>
__device__ __forceinline__ T put_rounded(float f, int sr, uint64_t pos, uint64_t base, uint32_t key)
{
    return sr ? Sr<T>::put(f, sr_bits(pos, base, key)) : Io<T>::put(f);
}

// a stochastic store of one 16-byte vector of V values starting at the
// (even) padded position pos0: one hash per voxel pair
template <typename T>
__device__ __forceinline__ void st_sr(T *p, const float (&r)[Io<T>::VEC], uint64_t pos0, uint64_t base, uint32_t key)
{
    constexpr int V = Io<T>::VEC;
    if constexpr (V == 8) {
        uint4 v;
        uint32_t *w32 = reinterpret_cast<uint32_t *>(&v);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t w = sr_word(pos0 + 2 * k, base, key);
            const T lo = Sr<T>::put(r[2 * k], w & 0xffffu), hi = Sr<T>::put(r[2 * k + 1], w >> 16);
            w32[k] = (uint32_t)*reinterpret_cast<const unsigned short *>(&lo) |
                     ((uint32_t)*reinterpret_cast<const unsigned short *>(&hi) << 16);
        }
        __stcs(reinterpret_cast<uint4 *>(p), v);
    } else {
        Io<T>::st(p, r);
    }
}

template <int VEC> __device__ inline void ld_code(const uint8_t *p, uint8_t (&c)[VEC]);
template <> __device__ inline void ld_code<4>(const uint8_t *p, uint8_t (&c)[4])
{
    const uchar4 v = __ldcs(reinterpret_cast<const uchar4 *>(p));
    c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
}
template <> __device__ inline void ld_code<8>(const uint8_t *p, uint8_t (&c)[8])
{
    const uint2 v = __ldcs(reinterpret_cast<const uint2 *>(p));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        c[i] = (v.x >> (8 * i)) & 0xff;
        c[4 + i] = (v.y >> (8 * i)) & 0xff;
    }
}

__device__ __forceinline__ float pick(uint8_t code, uint8_t bit, float centre, float nb)
{
    return (code & bit) ? centre : nb;
}

// simulator_gpu.cu:70-88 with the contractions of the reference build.
__device__ __forceinline__ float leapfrog(uint8_t c, float ce, float xp, float xm, float yp, float ym, float zp,
                                          float zm, float qv, float c2dt2, float inv_h2)
{
    float s = pick(c, W_XP, ce, xp);
    s = __fadd_rn(s, pick(c, W_XM, ce, xm));
    s = __fadd_rn(s, pick(c, W_YP, ce, yp));
    s = __fadd_rn(s, pick(c, W_YM, ce, ym));
    s = __fadd_rn(s, pick(c, W_ZP, ce, zp));
    s = __fadd_rn(s, pick(c, W_ZM, ce, zm));
    const float lap = __fmul_rn(__fmaf_rn(-6.0f, ce, s), inv_h2);
    const float t = __fsub_rn(__fmul_rn(2.0f, ce), qv);
    return __fmaf_rn(c2dt2, lap, t);
}

// the same update for an air voxel without wall neighbours (code 0): no
// selects; bit-identical to leapfrog(0, ...)
__device__ __forceinline__ float leapfrog_air(float ce, float xp, float xm, float yp, float ym, float zp, float zm,
                                              float qv, float c2dt2, float inv_h2)
{
    float s = __fadd_rn(xp, xm);
    s = __fadd_rn(s, yp);
    s = __fadd_rn(s, ym);
    s = __fadd_rn(s, zp);
    s = __fadd_rn(s, zm);
    const float lap = __fmul_rn(__fmaf_rn(-6.0f, ce, s), inv_h2);
    const float t = __fsub_rn(__fmul_rn(2.0f, ce), qv);
    return __fmaf_rn(c2dt2, lap, t);
}

// two air voxels at once with the packed FP32 instructions of sm_100, whose
// components round exactly like the scalar __fadd_rn / __fmul_rn /
// __fmaf_rn: bit-identical to two leapfrog_air calls.  The first sum
// (xp + xm) comes in as x2: its operands straddle the register pairs of a
// loaded vector, so it is two scalar adds.  2*ce is exact, so
// fma(2, ce, -qv) rounds like fsub(2*ce, qv) (they part only where 2*ce
// overflows).
__device__ __forceinline__ float2 leapfrog_air2(float2 ce, float2 x2, float2 yp, float2 ym, float2 zp, float2 zm,
                                                float2 qv, float2 c2dt2, float2 inv_h2)
{
    float2 s = __fadd2_rn(x2, yp);
    s = __fadd2_rn(s, ym);
    s = __fadd2_rn(s, zp);
    s = __fadd2_rn(s, zm);
    const float2 lap = __fmul2_rn(__ffma2_rn(make_float2(-6.0f, -6.0f), ce, s), inv_h2);
    const float2 t = __ffma2_rn(make_float2(2.0f, 2.0f), ce, __fmul2_rn(qv, make_float2(-1.0f, -1.0f)));
    return __ffma2_rn(c2dt2, lap, t);
}

// simulator_gpu.cu:126-148: biquad sections in series on d = p - p^{n-1}
// (b0*in + b1*s0 contracted to fma(b0, in, b1*s0) as the reference build
// does), then p+ -= K*(0.1*y + 0.9*d)*0.4 (times the sponge weight) in
// double, or the centered form of the same correction.

// the correction, given the cascade output y (double precision)
__device__ __forceinline__ float correct(const StepArgs &a, float r, float d, float y, float qv, float wf)
{
    const double w = (double)wf;
    if (a.form == VIRS_BOUNDARY_REFERENCE) {
        const double t = __fma_rn((double)y, a.mix_y, __dmul_rn((double)d, a.mix_d));
        const double u = __dmul_rn(__dmul_rn(__dmul_rn(a.K, t), a.gain), w);
        return __double2float_rn(__dsub_rn((double)r, u));
    }
    // centered: the direct damping term at (p+ - p-)/2, solved for p+
    const double kgw = __dmul_rn(__dmul_rn(a.K, a.gain), w);
    const double ac = __dmul_rn(__dmul_rn(kgw, a.mix_d), 0.5);
    const double num = __dadd_rn(__dsub_rn((double)r, __dmul_rn(kgw, __dmul_rn((double)y, a.mix_y))),
                                 __dmul_rn(ac, (double)qv));
    return __double2float_rn(__ddiv_rn(num, __dadd_rn(1.0, ac)));
}

// Filter states.  In a cascade the output of section q is the input of
// section q+1, so the two past outputs a DF1 section keeps (y[n-1], y[n-2])
// are the two past inputs of the next one: S sections need 2(S+1) values,
// X_q[n-1] and X_q[n-2] for the input X_0 = p - p^{n-1} and the outputs
// X_{q+1} = y_q (entry 2q holds X_q[n-1], 2q+1 holds X_q[n-2]).  This is
// the reference's four states per section (simulator_gpu.cu:126-146)
// without the copies, so every value, and the result, is the same.  They
// are stored in groups of four entries per slot (state_index in
// internal.hpp): one 16-byte load and store per group.

// up to MAXS sections, fully unrolled, in two parts so that a caller can
// issue the loads of a voxel before any arithmetic: bload reads the
// material, the weight and every state of a slot; bcompute reads the
// coefficients (they depend on the material), runs the cascade, writes the
// states and returns the corrected value.
template <int MAXS> struct BState {
    static constexpr int NG = (2 * (MAXS + 1) + 3) / 4; // vector groups
    uint32_t m;
    float wf;
    float h[4 * NG];                                    // entry e = 2q + j
};

template <int MAXS> __device__ __forceinline__ void bload(const StepArgs &a, uint64_t slot, BState<MAXS> &b)
{
    const uint32_t ng = (2u * (a.nsec + 1u) + 3u) / 4u;
    const float4 *st = reinterpret_cast<const float4 *>(a.state) + slot;
    b.m = __ldg(a.bmat + slot);
    b.wf = __ldg(a.bw + slot);
#pragma unroll
    for (int g = 0; g < BState<MAXS>::NG; ++g)
        if ((uint32_t)g < ng) {
            const float4 v = st[(uint64_t)g * a.nb];
            b.h[4 * g] = v.x;
            b.h[4 * g + 1] = v.y;
            b.h[4 * g + 2] = v.z;
            b.h[4 * g + 3] = v.w;
        }
}

template <int MAXS>
__device__ __forceinline__ float bcompute(const StepArgs &a, float r, float ce, float qv, uint64_t slot,
                                          const BState<MAXS> &b)
{
    const uint32_t ns = a.nsec, ng = (2u * (ns + 1u) + 3u) / 4u;
    float4 *st = reinterpret_cast<float4 *>(a.state_out ? a.state_out : a.state) + slot;
    const float *kc = a.coef + (uint64_t)b.m * ns * 5;
    const float d = __fsub_rn(ce, qv);
    float in = d, last = b.h[0];
    float nv[4 * BState<MAXS>::NG]; // the states after this step
#pragma unroll
    for (int e = 0; e < 4 * BState<MAXS>::NG; ++e) nv[e] = 0.f;
#pragma unroll
    for (int q = 0; q < MAXS; ++q) {
        if (q < (int)ns) {
            const float *kq = kc + 5 * q;
            float y = __fmaf_rn(__ldg(kq), in, __fmul_rn(__ldg(kq + 1), b.h[2 * q]));
            y = __fmaf_rn(__ldg(kq + 2), b.h[2 * q + 1], y);
            y = __fmaf_rn(-__ldg(kq + 3), b.h[2 * q + 2], y);
            y = __fmaf_rn(-__ldg(kq + 4), b.h[2 * q + 3], y);
            nv[2 * q] = in;
            nv[2 * q + 1] = b.h[2 * q];
            in = y;
            last = b.h[2 * q + 2];
        }
    }
    // the history of the last output, entries 2S and 2S+1
#pragma unroll
    for (int q = 0; q <= MAXS; ++q)
        if (q == (int)ns) {
            nv[2 * q] = in;
            nv[2 * q + 1] = last;
        }
#pragma unroll
    for (int g = 0; g < BState<MAXS>::NG; ++g)
        if ((uint32_t)g < ng) st[(uint64_t)g * a.nb] = make_float4(nv[4 * g], nv[4 * g + 1], nv[4 * g + 2], nv[4 * g + 3]);
    return correct(a, r, d, in, qv, b.wf);
}

// any number of sections
__device__ __noinline__ float boundary_loop(const StepArgs &a, float r, float ce, float qv, uint64_t slot)
{
    const float d = __fsub_rn(ce, qv);
    float in = d;
    const uint64_t nb = a.nb;
    const float *kc = a.coef + (uint64_t)__ldg(a.bmat + slot) * a.nsec * 5;
    const float *si = a.state;
    float *st = a.state_out ? a.state_out : a.state;
    float x1 = si[state_index(0, slot, nb)], x2 = si[state_index(1, slot, nb)];
    for (uint32_t q = 0; q < a.nsec; ++q, kc += 5) {
        const float y1 = si[state_index(2 * q + 2, slot, nb)], y2 = si[state_index(2 * q + 3, slot, nb)];
        float y = __fmaf_rn(__ldg(kc), in, __fmul_rn(__ldg(kc + 1), x1));
        y = __fmaf_rn(__ldg(kc + 2), x2, y);
        y = __fmaf_rn(-__ldg(kc + 3), y1, y);
        y = __fmaf_rn(-__ldg(kc + 4), y2, y);
        st[state_index(2 * q, slot, nb)] = in;
        st[state_index(2 * q + 1, slot, nb)] = x1;
        in = y;
        x1 = y1;
        x2 = y2;
    }
    st[state_index(2 * a.nsec, slot, nb)] = in;
    st[state_index(2 * a.nsec + 1, slot, nb)] = x1;
    return correct(a, r, d, in, qv, __ldg(a.bw + slot));
}

} // namespace
} // namespace step
} // namespace virs
