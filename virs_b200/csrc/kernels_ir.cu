// IR post-processing on the GPU: the receiver traces recorded at the
// simulation rate 1/dt become output-rate signals.
//
// The reference does this on the host after the step loop
// (simulator.cpp:1029-1080): a library resampler (kfr) to 48 kHz, then
// division by the peak magnitude.  Here, per receiver channel:
//   k_ir_sos       the anti-alias cascade of second-order sections in FP64,
//                  transposed direct form II (the recursion of
//                  src/util/downsampling_filter_iir.cpp:210-240), as a
//                  systolic warp: lane s owns section s and its two states,
//                  and at tick t it filters sample t - s, taking its input
//                  from lane s-1's output of the previous tick (a shuffle);
//                  the last lane's output is the filtered sample
//   k_ir_resample  linear interpolation at k / rate (simulator.cpp:1046-1057),
//                  then, if asked, division by the channel's peak
// Every product and sum is written with _rn intrinsics in the CPU
// recursion's order (no contraction), so the result is bit for bit the
// oracle's.
#include "internal.hpp"

namespace virs {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int CHUNK = 1024; // input samples staged per round of ticks

__global__ void __launch_bounds__(32) k_ir_sos(const float *__restrict in, uint64_t in_stride, uint64_t len,
                                               const double *__restrict sos, int ns, float *__restrict out,
                                               uint64_t out_stride)
{
    __shared__ float xin[CHUNK];
    const int lane = threadIdx.x;
    const float *x = in + blockIdx.x * in_stride;
    float *y = out + blockIdx.x * out_stride;
    double b0 = 0, b1 = 0, b2 = 0, a1 = 0, a2 = 0;
    if (lane < ns) {
        const double *s = sos + 6 * lane;
        b0 = s[0]; b1 = s[1]; b2 = s[2]; a1 = s[4]; a2 = s[5];
    }
    double z1 = 0.0, z2 = 0.0, last = 0.0; // `last`: this lane's output of the previous tick
    const uint64_t ticks = len + (uint64_t)ns - 1;
    for (uint64_t c0 = 0; c0 < ticks; c0 += CHUNK) {
        __syncwarp();
        for (int i = lane; i < CHUNK; i += 32) {
            const uint64_t t = c0 + (uint64_t)i;
            xin[i] = t < len ? x[t] : 0.f;
        }
        __syncwarp();
        const int m = ticks - c0 < (uint64_t)CHUNK ? (int)(ticks - c0) : CHUNK;
        for (int i = 0; i < m; ++i) {
            const uint64_t t = c0 + (uint64_t)i;
            const double up = __shfl_up_sync(FULL, last, 1);
            const double v = lane == 0 ? (double)xin[i] : up;
            if (lane < ns && t >= (uint64_t)lane && t - (uint64_t)lane < len) {
                const double yo = __dadd_rn(__dmul_rn(b0, v), z1);
                const double n1 = __dadd_rn(__dsub_rn(__dmul_rn(b1, v), __dmul_rn(a1, yo)), z2);
                const double n2 = __dsub_rn(__dmul_rn(b2, v), __dmul_rn(a2, yo));
                z1 = n1;
                z2 = n2;
                last = yo;
                if (lane == ns - 1) y[t - (uint64_t)lane] = __double2float_rn(yo);
            }
        }
    }
}

constexpr int RB = 256;

__global__ void __launch_bounds__(RB) k_ir_resample(const float *__restrict in, uint64_t in_stride, uint64_t len,
                                                    double sim_rate, float rate, float *__restrict out,
                                                    uint64_t out_len, int normalize)
{
    __shared__ float red[RB / 32];
    const float *f = in + blockIdx.x * in_stride;
    float *o = out + blockIdx.x * out_len;
    float peak = 0.f;
    for (uint64_t k = threadIdx.x; k < out_len; k += RB) {
        const float t = __fdiv_rn((float)k, rate);
        const float index = __double2float_rn(__dmul_rn((double)t, sim_rate));
        uint64_t lo = (uint64_t)floorf(index);
        if (lo >= len) lo = len - 1;
        const uint64_t hi = lo + 1 < len ? lo + 1 : lo;
        const float frac = __fsub_rn(index, (float)lo);
        const float v = __fadd_rn(__fmul_rn(f[lo], __fsub_rn(1.f, frac)), __fmul_rn(f[hi], frac));
        o[k] = v;
        peak = fmaxf(peak, fabsf(v));
    }
    if (!normalize) return;
    for (int s = 16; s > 0; s >>= 1) peak = fmaxf(peak, __shfl_xor_sync(FULL, peak, s));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = peak;
    __syncthreads();
    peak = 0.f;
    for (int w = 0; w < RB / 32; ++w) peak = fmaxf(peak, red[w]);
    if (!(peak > 0.f)) return; // a silent channel stays zero
    for (uint64_t k = threadIdx.x; k < out_len; k += RB) o[k] = __fdiv_rn(o[k], peak);
}

// Band-limited resampling with a Kaiser-windowed sinc: output sample k is
// at input position t = k * fs_in / rate; y_k = sum over the input samples
// n with |t - n| < half of x[n] * 2 fc sinc(2 fc (t - n)) * w(t - n), with
// fc = cutoff * min(fs_in, rate) / 2 / fs_in (cycles per input sample),
// sinc(u) = sin(pi u) / (pi u) and the Kaiser window
// w(tau) = I0(beta sqrt(1 - (tau / half)^2)) / I0(beta).  I0 is summed from
// its power series, sum_k ((x / 2)^k / k!)^2.  FP64 throughout; one thread
// per output sample of one channel (blockIdx.y).
__device__ double bessel_i0(double x)
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

__global__ void __launch_bounds__(RB) k_ir_sinc(const float *__restrict in, uint64_t in_stride, uint64_t len,
                                                double step_ratio, double fc2, int half, double beta, double i0b,
                                                float *__restrict out, uint64_t out_len, uint32_t *__restrict peak)
{
    const uint64_t k = (uint64_t)blockIdx.x * RB + threadIdx.x;
    if (k >= out_len) return;
    const float *f = in + blockIdx.y * in_stride;
    const double t = (double)k * step_ratio;
    const double n0 = fmax(0.0, ceil(t - (double)half)), n1 = fmin((double)len - 1.0, floor(t + (double)half));
    double acc = 0.0;
    for (double n = n0; n <= n1; n += 1.0) {
        const double tau = t - n, u = tau / (double)half;
        if (!(fabs(u) < 1.0)) continue;
        const double w = bessel_i0(beta * sqrt(1.0 - u * u)) / i0b;
        const double x = fc2 * tau;
        const double sc = x == 0.0 ? 1.0 : sin(M_PI * x) / (M_PI * x);
        acc += (double)f[(uint64_t)n] * (fc2 * sc * w);
    }
    const float v = (float)acc;
    out[blockIdx.y * out_len + k] = v;
    if (peak) atomicMax(peak + blockIdx.y, __float_as_uint(fabsf(v))); // non-negative floats order as integers
}

__global__ void k_ir_normalize(float *__restrict out, uint64_t out_len, const uint32_t *__restrict peak)
{
    const uint64_t k = (uint64_t)blockIdx.x * RB + threadIdx.x;
    const float p = __uint_as_float(peak[blockIdx.y]);
    if (k < out_len && p > 0.f) out[blockIdx.y * out_len + k] = __fdiv_rn(out[blockIdx.y * out_len + k], p);
}

} // namespace

cudaError_t launch_ir_sinc(const float *in, uint64_t in_stride, uint64_t len, double fs_in, double rate, int half,
                           double beta, double cutoff, float *out, uint64_t out_len, uint32_t *peak, uint32_t channels,
                           cudaStream_t s)
{
    if (!channels || !out_len || !len) return cudaSuccess;
    const double fc2 = cutoff * fmin(fs_in, rate) / fs_in;        // 2 fc
    double i0b = 1.0, t = 1.0;
    for (int k = 1; k < 500; ++k) {                                // I0(beta), as the kernel sums it
        t = t * (0.25 * beta * beta) / ((double)k * (double)k);
        i0b = i0b + t;
        if (t < 1e-17 * i0b) break;
    }
    const dim3 g((unsigned)((out_len + RB - 1) / RB), channels);
    if (peak) {
        cudaError_t e = cudaMemsetAsync(peak, 0, channels * sizeof(uint32_t), s);
        if (e != cudaSuccess) return e;
    }
    k_ir_sinc<<<g, RB, 0, s>>>(in, in_stride, len, fs_in / rate, fc2, half, beta, i0b, out, out_len, peak);
    if (peak) k_ir_normalize<<<g, RB, 0, s>>>(out, out_len, peak);
    return cudaGetLastError();
}

cudaError_t launch_ir_sos(const float *in, uint64_t in_stride, uint64_t len, const double *sos, int ns, float *out,
                          uint64_t out_stride, uint32_t channels, cudaStream_t s)
{
    if (!channels || !len) return cudaSuccess;
    k_ir_sos<<<channels, 32, 0, s>>>(in, in_stride, len, sos, ns, out, out_stride);
    return cudaGetLastError();
}

cudaError_t launch_ir_resample(const float *in, uint64_t in_stride, uint64_t len, double sim_rate, float rate,
                               float *out, uint64_t out_len, int normalize, uint32_t channels, cudaStream_t s)
{
    if (!channels || !out_len || !len) return cudaSuccess;
    k_ir_resample<<<channels, RB, 0, s>>>(in, in_stride, len, sim_rate, rate, out, out_len, normalize);
    return cudaGetLastError();
}

} // namespace virs
