// Replays the reference's own sequence of dispatch calls (Simulator::loadObj
// and Simulator::simulate, src/simulator/simulator.cpp) through the binding
// virs_b200/integration/virs_dispatch.cpp, on a voxelised grid read from a
// file, and writes what the reference would hold afterwards.
//
//   dispatch_replay <in> <out>
//   in : u64 nx, ny, nz, steps, rx, ry, rz; f32 h; u8 flags[nx*ny*nz]
//        (the host triangle sweep's flags, 0/1/3)
//   out: u8 flags[N] after buildSpongeLayer; u64 nb; u32 boundary list[nb]
//        (built on the host as simulator.cpp:572-605 does); u64 steps run;
//        f32 p_audio_output[steps]; f32 p_curr[N] after the run
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "simulator_dispatch.h"
#include "virs.h"
#include "virs_dispatch.h"

namespace {

template <typename T> bool get(FILE *f, T *v, std::size_t n = 1) { return std::fread(v, sizeof(T), n, f) == n; }
template <typename T> void put(FILE *f, const T *v, std::size_t n = 1) { std::fwrite(v, sizeof(T), n, f); }

int run(const char *in_path, const char *out_path)
{
    FILE *in = std::fopen(in_path, "rb");
    if (!in) return 2;
    uint64_t hdr[7];
    float h = 0.f;
    if (!get(in, hdr, 7) || !get(in, &h)) return 2;
    const std::size_t nx = hdr[0], ny = hdr[1], nz = hdr[2], steps = hdr[3];
    std::vector<uint8_t> voxelised(nx * ny * nz);
    if (!get(in, voxelised.data(), voxelised.size())) return 2;
    std::fclose(in);

    // Simulator::loadObj, forSimulation (simulator.cpp:337-341)
    VectorSpace space(nx, ny, nz, AudioFile<float>(), h);
    Grid &grid = space.getGrid();
    grid.num_filter_sections = 3;
    grid.allocated_filter_memory = false;
    fdtd_setup(&space);
    // the triangle sweep writes the host flags (simulator.cpp:396-452)
    std::memcpy(grid.flags, voxelised.data(), voxelised.size());
    buildSpongeLayer(&space);                       // :469
    grid.boundary_indices_size = 0;                 // :472
    updateGPUFromGrid(&space);                      // :474
    // normals on the host from the classified flags (:480-566): bit set for
    // each face neighbour whose flag is 0 (+x 1, -x 2, +y 4, -y 8, +z 16, -z 32)
    for (std::size_t k = 1; k + 1 < nz; ++k)
        for (std::size_t j = 1; j + 1 < ny; ++j)
            for (std::size_t i = 1; i + 1 < nx; ++i) {
                uint8_t m = 0;
                m |= grid.flags[grid.idx(i + 1, j, k)] == 0 ? 1 : 0;
                m |= grid.flags[grid.idx(i - 1, j, k)] == 0 ? 2 : 0;
                m |= grid.flags[grid.idx(i, j + 1, k)] == 0 ? 4 : 0;
                m |= grid.flags[grid.idx(i, j - 1, k)] == 0 ? 8 : 0;
                m |= grid.flags[grid.idx(i, j, k + 1)] == 0 ? 16 : 0;
                m |= grid.flags[grid.idx(i, j, k - 1)] == 0 ? 32 : 0;
                grid.normals[grid.idx(i, j, k)] = m;
            }
    uploadNormalsToGPU(&space);                     // :569
    // boundary list, interior flag-2 voxels in ascending order (:572-605)
    std::vector<uint32_t> blist;
    for (std::size_t k = 1; k + 1 < nz; ++k)
        for (std::size_t j = 1; j + 1 < ny; ++j)
            for (std::size_t i = 1; i + 1 < nx; ++i)
                if (grid.flags[grid.idx(i, j, k)] == 2) blist.push_back((uint32_t)grid.idx(i, j, k));
    grid.boundary_indices_size = blist.size();
    grid.boundary_indices = blist.data();
    allocFilterStates(&space);                      // :610
    uploadBoundaryIndicesToGPU(&space);             // :635
    virs_dispatch_set_receiver(&space, hdr[4], hdr[5], hdr[6]);

    // Simulator::simulate (simulator.cpp:933-1025)
    const double hd = space.h;
    const double dt = 0.5 * hd / (343.0 * std::sqrt(3.0));
    const double simulation_fs = 1.f / dt;
    allocFilterCoeffs(&space, 1);                   // :955
    if (virs_design_highpass((float)simulation_fs, 440.f, 0.1f, 1.f, grid.biquad_coeffs) != VIRS_OK) return 3;
    uploadFilterCoeffsToGPU(&space);                // :964
    fdtd_start_simulation(&space, steps);           // :973
    updateCurrentGridFromGPU(&space);               // :975
    std::size_t ran = 0;
    for (std::size_t i = 0; i < steps; ++i) {       // :981-1025, doSimulationStep :921-931
        const bool keep = fdtd_step(&space, (unsigned)i);
        ++ran;
        if (!keep) break;
    }
    updateCurrentGridFromGPU(&space);               // :1027

    FILE *out = std::fopen(out_path, "wb");
    if (!out) return 2;
    put(out, grid.flags, grid.size);
    const uint64_t nb = blist.size(), nran = ran;
    put(out, &nb);
    put(out, blist.data(), blist.size());
    put(out, &nran);
    put(out, grid.p_audio_output, steps);
    put(out, grid.p_curr, grid.size);
    std::fclose(out);
    grid.boundary_indices = nullptr;
    fdtd_cleanup(&space);                           // ~Simulator, :909
    return 0;
}

} // namespace

int main(int argc, char **argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: dispatch_replay <in> <out>\n");
        return 2;
    }
    try {
        return run(argv[1], argv[2]);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 4;
    }
}
