// Small kernels around the step: the FP64 energy monitor, the sphere
// initial condition, and packing between the padded, scaled storage and the
// reference layout in FP32.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "internal.hpp"

namespace virs {
namespace {

__device__ __forceinline__ float tof(float v) { return v; }
__device__ __forceinline__ float tof(__half v) { return __half2float(v); }
__device__ __forceinline__ float tof(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename T> __device__ __forceinline__ T fromf(float v);
template <> __device__ __forceinline__ float fromf<float>(float v) { return v; }
template <> __device__ __forceinline__ __half fromf<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 fromf<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

constexpr int EB = 256; // energy block size

// Discrete energy of the lossless scheme (FP64):
//   E = sum_active (p - q)^2 + lambda2 * sum_links (p_i - p_j)(q_i - q_j)
// Active voxels are the ones the leapfrog updates (air and boundary).  A link
// joins an active voxel to a face neighbour that is not a wall (the wall
// mask of its code says which are); links between two active voxels are
// counted once (forward direction), links to fixed voxels (border, hard
// source) in both directions.  Per-block partial sums go to partial[].
template <typename T>
__global__ void __launch_bounds__(EB) k_energy(const T *__restrict p, const T *__restrict q, const uint8_t *__restrict code,
                                               uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px, double lambda2,
                                               double *__restrict partial)
{
    __shared__ double sh[EB / 32];
    const size_t sy = px, sz = (size_t)px * ny, n = sz * nz;
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * EB + threadIdx.x; i < n; i += (size_t)gridDim.x * EB) {
        const uint8_t c = code[i];
        if (c >= CODE_HARD) continue;
        const double pi = tof(p[i]), qi = tof(q[i]);
        double pot = 0.0;
        const size_t off[3] = {1, sy, sz};
        const uint8_t fw[3] = {W_XP, W_YP, W_ZP}, bw[3] = {W_XM, W_YM, W_ZM};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (!(c & fw[a])) {
                const size_t j = i + off[a];
                pot += (pi - (double)tof(p[j])) * (qi - (double)tof(q[j]));
            }
            if (!(c & bw[a])) {
                const size_t j = i - off[a];
                if (code[j] >= CODE_HARD) pot += (pi - (double)tof(p[j])) * (qi - (double)tof(q[j]));
            }
        }
        acc += (pi - qi) * (pi - qi) + lambda2 * pot;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < EB / 32; ++w) s += sh[w];
        partial[blockIdx.x] = s;
    }
}

// fixed-order sum of the partials into partial[nblocks]
__global__ void k_energy_final(double *partial, int nblocks, double scale2)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += partial[b];
        partial[nblocks] = s * scale2;
    }
}

// init_sphere.cu:4-25 restricted to interior voxels (border voxels stay 0)
template <typename T>
__global__ void k_sphere(T *p, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px, uint64_t cx, uint64_t cy,
                         uint64_t cz, uint64_t r2, float value, int init)
{
    const uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x == 0 || y == 0 || z == 0 || x + 1 >= nx || y + 1 >= ny || z + 1 >= nz) return;
    const uint64_t dx = x > cx ? x - cx : cx - x, dy = y > cy ? y - cy : cy - y, dz = z > cz ? z - cz : cz - z;
    const size_t i = ((size_t)z * ny + y) * px + x;
    if (dx * dx + dy * dy + dz * dz <= r2) p[i] = fromf<T>(value);
    else if (init) p[i] = fromf<T>(0.f);
}

template <typename T>
__global__ void k_pack(const T *f, float *out, uint32_t nx, uint32_t ny, uint32_t px, float inv_scale)
{
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    out[((size_t)z * ny + y) * nx + x] = __fmul_rn(tof(f[((size_t)z * ny + y) * px + x]), inv_scale);
}

template <typename T>
__global__ void k_unpack(const float *in, T *f, uint32_t nx, uint32_t ny, uint32_t px, float scale)
{
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    f[((size_t)z * ny + y) * px + x] = fromf<T>(__fmul_rn(in[((size_t)z * ny + y) * nx + x], scale));
}

template <typename F> cudaError_t by_storage(int storage, F &&f)
{
    switch (storage) {
    case VIRS_STORAGE_F16: return f(__half());
    case VIRS_STORAGE_BF16: return f(__nv_bfloat16());
    default: return f(float());
    }
}

} // namespace

cudaError_t launch_energy(int storage, const void *p, const void *q, const uint8_t *code, uint32_t nx, uint32_t ny,
                          uint32_t nz, uint32_t px, double lambda2, double inv_scale2, double *partial, int nblocks,
                          cudaStream_t s)
{
    return by_storage(storage, [&](auto t) {
        using T = decltype(t);
        k_energy<T><<<nblocks, EB, 0, s>>>((const T *)p, (const T *)q, code, nx, ny, nz, px, lambda2, partial);
        k_energy_final<<<1, 32, 0, s>>>(partial, nblocks, inv_scale2);
        return cudaGetLastError();
    });
}

cudaError_t launch_sphere(int storage, void *p, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px, uint64_t cx,
                          uint64_t cy, uint64_t cz, uint64_t r, float value, int init, cudaStream_t s)
{
    return by_storage(storage, [&](auto t) {
        using T = decltype(t);
        k_sphere<T><<<dim3((nx + 127) / 128, ny, nz), 128, 0, s>>>((T *)p, nx, ny, nz, px, cx, cy, cz, r * r, value,
                                                                   init);
        return cudaGetLastError();
    });
}

cudaError_t launch_pack(int storage, const void *field, float *out, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px,
                        float inv_scale, cudaStream_t s)
{
    return by_storage(storage, [&](auto t) {
        using T = decltype(t);
        k_pack<T><<<dim3((nx + 127) / 128, ny, nz), 128, 0, s>>>((const T *)field, out, nx, ny, px, inv_scale);
        return cudaGetLastError();
    });
}

cudaError_t launch_unpack(int storage, const float *in, void *field, uint32_t nx, uint32_t ny, uint32_t nz,
                          uint32_t px, float scale, cudaStream_t s)
{
    return by_storage(storage, [&](auto t) {
        using T = decltype(t);
        k_unpack<T><<<dim3((nx + 127) / 128, ny, nz), 128, 0, s>>>(in, (T *)field, nx, ny, px, scale);
        return cudaGetLastError();
    });
}

} // namespace virs
