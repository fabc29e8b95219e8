// Harness that runs the reference's own CUDA kernels (TEST INFRASTRUCTURE).
//
// oracle/Makefile cuts the self-contained kernel ranges out of the reference
// tree into _ref/gpu_extract.inc:
//   src/simulator/simulator_gpu.cu:9-180  constants, fdtd_kernel,
//                                         fdtd_kernel_boundary_biquad,
//                                         fdtd_kernel_rigid_walls
//   src/simulator/sponge_kernel.cu:5-62   N, EPS, spongeKernel
// and compiles them with the reference's CUDA flags (--use_fast_math).  The
// host driver below follows fdtd_gpu_step (simulator_gpu.cu:184-300) and
// buildSpongeLayerGPU (sponge_kernel.cu:65-99): the same constants, launch
// shapes, source schedule, launch order and pointer rotation.  It differs in
// two ways only: receivers are a caller-given list instead of the fixed
// voxel (334,225,270), and constants are uploaded on every run instead of
// once per process.  The output is used to generate golden vectors.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cuda_runtime.h>

#include "gpu_extract.inc"

namespace {

__global__ void probe_constants(float *out)
{
    // the boundary scale exactly as fdtd_kernel_boundary_biquad evaluates it
    // (simulator_gpu.cu:147), compiled with the same flags
    out[0] = (d_c_sound * d_dt) / d_dx * 0.95f;
    // the rigid-wall update's l2 as fdtd_kernel_rigid_walls evaluates it
    // (simulator_gpu.cu:165)
    out[1] = (d_c_sound * d_dt / d_dx) * (d_c_sound * d_dt / d_dx);
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

} // namespace

#define RCHECK(x)                                  \
    do {                                           \
        cudaError_t e_ = (x);                      \
        if (e_ != cudaSuccess) return (int)e_;     \
    } while (0)

extern "C" {

__attribute__((visibility("default"))) int ref_gpu_sponge(uint64_t nx, uint64_t ny, uint64_t nz,
                                                          const uint8_t *flags_in, uint8_t *flags_out)
{
    const size_t n = nx * ny * nz;
    DevBuf din, dout, dabs;
    RCHECK(cudaMalloc(&din.p, n));
    RCHECK(cudaMalloc(&dout.p, n));
    RCHECK(cudaMalloc(&dabs.p, n * sizeof(float)));
    RCHECK(cudaMemcpy(din.p, flags_in, n, cudaMemcpyHostToDevice));
    RCHECK(cudaMemcpy(dout.p, flags_in, n, cudaMemcpyHostToDevice));
    dim3 B(8, 8, 8);
    dim3 G((unsigned)((nx + 7) / 8), (unsigned)((ny + 7) / 8), (unsigned)((nz + 7) / 8));
    spongeKernel<<<G, B>>>((const uint8_t *)din.p, (uint8_t *)dout.p, (float *)dabs.p, nx, ny, nz);
    RCHECK(cudaGetLastError());
    RCHECK(cudaDeviceSynchronize());
    RCHECK(cudaMemcpy(flags_out, dout.p, n, cudaMemcpyDeviceToHost));
    return 0;
}

// consts_out: dt, c2dt2, inv_h2 (host-computed and uploaded) and the device
// value of the boundary scale.
static int run_impl(uint64_t nx, uint64_t ny, uint64_t nz, float h, const uint8_t *flags, const uint8_t *normals,
                    int rigid, const uint32_t *bidx, uint64_t nb, const float *coeffs5, uint32_t steps, uint32_t nrcv,
                    const uint64_t *rcv, float *ir, float *p_final, float *consts_out);

__attribute__((visibility("default"))) int ref_gpu_run(uint64_t nx, uint64_t ny, uint64_t nz, float h,
                                                       const uint8_t *flags, const uint32_t *bidx, uint64_t nb,
                                                       const float *coeffs5, uint32_t steps, uint32_t nrcv,
                                                       const uint64_t *rcv, float *ir, float *p_final,
                                                       float *consts_out)
{
    return run_impl(nx, ny, nz, h, flags, nullptr, 0, bidx, nb, coeffs5, steps, nrcv, rcv, ir, p_final, consts_out);
}

// The same step with fdtd_kernel_rigid_walls launched between the interior
// and the filter kernels, as the commented launch at simulator_gpu.cu:280
// places it; `normals` is the air-neighbour mask of every voxel.
__attribute__((visibility("default"))) int ref_gpu_run_rigid(uint64_t nx, uint64_t ny, uint64_t nz, float h,
                                                             const uint8_t *flags, const uint8_t *normals,
                                                             const uint32_t *bidx, uint64_t nb,
                                                             const float *coeffs5, uint32_t steps, uint32_t nrcv,
                                                             const uint64_t *rcv, float *ir, float *p_final,
                                                             float *consts_out)
{
    return run_impl(nx, ny, nz, h, flags, normals, 1, bidx, nb, coeffs5, steps, nrcv, rcv, ir, p_final, consts_out);
}

} // extern "C"

static int run_impl(uint64_t nx, uint64_t ny, uint64_t nz, float h, const uint8_t *flags, const uint8_t *normals,
                    int rigid, const uint32_t *bidx, uint64_t nb, const float *coeffs5, uint32_t steps, uint32_t nrcv,
                    const uint64_t *rcv, float *ir, float *p_final, float *consts_out)
{
    const size_t n = nx * ny * nz;
    DevBuf bp[3], dflags, dnorm, dbidx, dstate, dcoef, dprobe;
    for (auto &b : bp) {
        RCHECK(cudaMalloc(&b.p, n * sizeof(float)));
        RCHECK(cudaMemset(b.p, 0, n * sizeof(float)));
    }
    RCHECK(cudaMalloc(&dflags.p, n));
    RCHECK(cudaMemcpy(dflags.p, flags, n, cudaMemcpyHostToDevice));
    RCHECK(cudaMalloc(&dnorm.p, n));
    if (normals) RCHECK(cudaMemcpy(dnorm.p, normals, n, cudaMemcpyHostToDevice));
    else RCHECK(cudaMemset(dnorm.p, 0, n));
    RCHECK(cudaMalloc(&dbidx.p, (nb ? nb : 1) * sizeof(uint32_t)));
    if (nb) RCHECK(cudaMemcpy(dbidx.p, bidx, nb * sizeof(uint32_t), cudaMemcpyHostToDevice));
    const size_t sections = 3; // simulator.cpp:339
    RCHECK(cudaMalloc(&dstate.p, (nb ? nb : 1) * sections * 4 * sizeof(float)));
    RCHECK(cudaMemset(dstate.p, 0, (nb ? nb : 1) * sections * 4 * sizeof(float)));
    RCHECK(cudaMalloc(&dcoef.p, 5 * sizeof(float)));
    RCHECK(cudaMemcpy(dcoef.p, coeffs5, 5 * sizeof(float), cudaMemcpyHostToDevice));
    RCHECK(cudaMalloc(&dprobe.p, 2 * sizeof(float)));

    // simulator_gpu.cu:191-209
    int iNx = (int)nx, iNy = (int)ny, iNz = (int)nz;
    size_t num_boundary_indices = nb;
    float c = 343.f;
    float dt = 0.5f * h / (c * std::sqrt(3.f));
    float c2_dt2 = c * c * dt * dt;
    float inv_h2 = 1.f / (h * h);
    RCHECK(cudaMemcpyToSymbol(d_Nx, &iNx, sizeof(int)));
    RCHECK(cudaMemcpyToSymbol(d_Ny, &iNy, sizeof(int)));
    RCHECK(cudaMemcpyToSymbol(d_Nz, &iNz, sizeof(int)));
    RCHECK(cudaMemcpyToSymbol(d_inv_h2, &inv_h2, sizeof(float)));
    RCHECK(cudaMemcpyToSymbol(d_c2_dt2, &c2_dt2, sizeof(float)));
    RCHECK(cudaMemcpyToSymbol(d_dt, &dt, sizeof(float)));
    RCHECK(cudaMemcpyToSymbol(d_c_sound, &c, sizeof(float)));
    RCHECK(cudaMemcpyToSymbol(d_dx, &h, sizeof(float)));
    RCHECK(cudaMemcpyToSymbol(d_num_boundary_indices, &num_boundary_indices, sizeof(size_t)));
    probe_constants<<<1, 1>>>((float *)dprobe.p);
    RCHECK(cudaGetLastError());
    if (consts_out) {
        consts_out[0] = dt;
        consts_out[1] = c2_dt2;
        consts_out[2] = inv_h2;
        RCHECK(cudaMemcpy(&consts_out[3], dprobe.p, sizeof(float), cudaMemcpyDeviceToHost));
        if (rigid) RCHECK(cudaMemcpy(&consts_out[4], (float *)dprobe.p + 1, sizeof(float), cudaMemcpyDeviceToHost));
    }

    float *d_prev = (float *)bp[0].p, *d_curr = (float *)bp[1].p, *d_next = (float *)bp[2].p;
    dim3 B(16, 4, 4);
    dim3 G((iNx + B.x - 1) / B.x, (iNy + B.y - 1) / B.y, (iNz + B.z - 1) / B.z);
    const size_t tpb = 256;
    const size_t nbb = (nb + tpb - 1) / tpb;
    for (uint32_t step = 0; step < steps; ++step) {
        float source_value = step < 10 ? 10.f : 0.f; // simulator_gpu.cu:214-218
        RCHECK(cudaMemcpyToSymbol(d_source_value, &source_value, sizeof(float)));
        fdtd_kernel<<<G, B>>>(d_prev, d_curr, d_next, (const uint8_t *)dflags.p, (const uint8_t *)dnorm.p);
        RCHECK(cudaGetLastError());
        RCHECK(cudaDeviceSynchronize());
        if (rigid && nbb)
            fdtd_kernel_rigid_walls<<<(unsigned)nbb, (unsigned)tpb>>>(d_curr, d_next, d_prev, (const uint8_t *)dflags.p,
                                                                       (const uint8_t *)dnorm.p,
                                                                       (const uint32_t *)dbidx.p);
        RCHECK(cudaGetLastError());
        RCHECK(cudaDeviceSynchronize());
        if (nbb)
            fdtd_kernel_boundary_biquad<<<(unsigned)nbb, (unsigned)tpb>>>(
                d_curr, d_next, d_prev, (float *)dcoef.p, sections, (float *)dstate.p, (const uint8_t *)dflags.p,
                (const uint8_t *)dnorm.p, (const uint32_t *)dbidx.p);
        RCHECK(cudaGetLastError());
        RCHECK(cudaDeviceSynchronize());
        // simulator_gpu.cu:292-293
        float *t = d_prev; d_prev = d_curr; d_curr = t;
        t = d_curr; d_curr = d_next; d_next = t;
        for (uint32_t r = 0; r < nrcv; ++r)
            RCHECK(cudaMemcpy(&ir[(size_t)r * steps + step], d_curr + rcv[r], sizeof(float),
                              cudaMemcpyDeviceToHost));
    }
    if (p_final) RCHECK(cudaMemcpy(p_final, d_curr, n * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}


