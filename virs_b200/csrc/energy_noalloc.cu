// virs_energy_noalloc: the FP64 energy monitor for callers that cannot
// allocate device memory.
//
// virs_energy allocates its reduction buffer with cudaMalloc on first use.
// Some callers cannot allow that: a real-time audio thread (cudaMalloc and
// cudaFree may synchronise the whole device and block), a host framework
// that owns all device memory through its own pool, or code that enqueues
// work while another thread is capturing a CUDA graph.  This variant keeps
// its scratch -- one partial sum per z plane -- in a file-scope device
// array of VIRS_ENERGY_MAX_PLANES doubles (64 KiB), which every GPU that
// loads the library holds until the process exits.  Grids with more planes
// are rejected with VIRS_E_ARG.
//
// The array's device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, the first time the entry
// point runs on it (make that first call before any stream capture).  All
// calls share the array: every call writes each partial it reads, so no
// state carries over, but calls whose work overlaps on the GPU race on it.
// The call records the handle's completion event on the stream it used, so
// virs_synchronize and virs_destroy wait for its reads of the fields.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <mutex>

#include "internal.hpp"

#define VIRS_EXPORT extern "C" __attribute__((visibility("default")))

namespace virs {
namespace {

constexpr int EB = 256;

static __device__ __align__(256) double g_plane_energy[VIRS_ENERGY_MAX_PLANES];

__device__ __forceinline__ float tof(float v) { return v; }
__device__ __forceinline__ float tof(__half v) { return __half2float(v); }
__device__ __forceinline__ float tof(__nv_bfloat16 v) { return __bfloat162float(v); }

// one block per interior plane; the same discrete energy as k_energy
// (kernels_misc.cu): kinetic term of active voxels plus lambda2 times the
// link terms (active-active links once, links to fixed voxels both ways,
// links to walls none)
template <typename T>
__global__ void __launch_bounds__(EB) k_energy_planes(const T *__restrict p, const T *__restrict q,
                                                     const uint8_t *__restrict code, uint32_t ny, uint32_t px,
                                                     double lambda2, double *__restrict plane_sums)
{
    __shared__ double sh[EB / 32];
    const uint32_t z = blockIdx.x + 1;
    const size_t sy = px, sz = (size_t)px * ny, base = (size_t)z * sz;
    double acc = 0.0;
    for (size_t o = threadIdx.x; o < sz; o += EB) {
        const size_t i = base + o;
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
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < EB / 32; ++w) t += sh[w];
        plane_sums[z] = t;
    }
}

// fixed-order sum over the interior planes into the caller's output
__global__ void k_energy_planes_sum(const double *__restrict plane_sums, uint32_t nz, double scale2, double *out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (uint32_t z = 1; z + 1 < nz; ++z) s += plane_sums[z];
        *out = s * scale2;
    }
}

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double *g_scratch[MAX_DEVICES] = {};

// device address of the static array on the current device (looked up once)
virs_status scratch_for(int dev, double **out)
{
    if (dev < 0 || dev >= MAX_DEVICES) return fail(VIRS_E_ARG, "virs_energy_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_plane_energy);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_plane_energy)");
        g_scratch[dev] = static_cast<double *>(p);
    }
    *out = g_scratch[dev];
    return VIRS_OK;
}

} // namespace
} // namespace virs

using namespace virs;

VIRS_EXPORT virs_status virs_energy_noalloc(virs_sim *sim, double *d_out, void *stream)
{
    if (!sim || !d_out) return fail(VIRS_E_ARG, "virs_energy_noalloc: null argument");
    EnergyInputs in{};
    VIRS_TRY(energy_inputs(sim, stream, &in));
    if (in.nz > VIRS_ENERGY_MAX_PLANES)
        return fail(VIRS_E_ARG, "virs_energy_noalloc: the grid has " + std::to_string(in.nz) +
                                    " planes; the static scratch holds " + std::to_string(VIRS_ENERGY_MAX_PLANES));
    double *scratch = nullptr;
    VIRS_TRY(scratch_for(in.device, &scratch));
    const unsigned planes = in.nz - 2;
    switch (in.storage) {
    case VIRS_STORAGE_F16:
        k_energy_planes<__half><<<planes, EB, 0, in.stream>>>((const __half *)in.p, (const __half *)in.q, in.code,
                                                               in.ny, in.px, in.lambda2, scratch);
        break;
    case VIRS_STORAGE_BF16:
        k_energy_planes<__nv_bfloat16><<<planes, EB, 0, in.stream>>>((const __nv_bfloat16 *)in.p,
                                                                      (const __nv_bfloat16 *)in.q, in.code, in.ny,
                                                                      in.px, in.lambda2, scratch);
        break;
    default:
        k_energy_planes<float><<<planes, EB, 0, in.stream>>>((const float *)in.p, (const float *)in.q, in.code, in.ny,
                                                              in.px, in.lambda2, scratch);
        break;
    }
    k_energy_planes_sum<<<1, 32, 0, in.stream>>>(scratch, in.nz, in.scale2, d_out);
    VIRS_CUDA(cudaGetLastError());
    // the handle's completion event now follows these reads of its fields, so
    // virs_synchronize and virs_destroy wait for them (also on a caller's
    // stream) before the fields can be freed
    VIRS_CUDA(cudaEventRecord(in.done, in.stream));
    return VIRS_OK;
}
