// virs_dispatch.cpp -- the reference's dispatch layer over libvirs_b200.
//
// Drop-in replacement for src/simulator/simulator_dispatch.cpp (with
// simulator_gpu.cpp and simulator_gpu.cu behind it) in the Snipet/VIRS tree:
// every function declared in src/simulator/simulator_dispatch.h:4-25 is
// implemented here over the C ABI of virs.h, for the order in which
// Simulator::loadObj and Simulator::simulate call them
// (src/simulator/simulator.cpp):
//
//   :341  fdtd_setup                 handle + the host arrays of the Grid
//         (the host triangle sweep fills grid.flags, simulator.cpp:396-452)
//   :469  buildSpongeLayer           upload the voxelised flags, classify on
//                                    the GPU (sponge, normals, boundary list),
//                                    classified flags back to grid.flags
//   :474  updateGPUFromGrid          flags unchanged: nothing to redo; the
//                                    host fields go to the device at the start
//   :569  uploadNormalsToGPU         normals were made by the classification
//   :610  allocFilterStates          host array as the reference's; the
//                                    device states belong to the handle
//   :635  uploadBoundaryIndicesToGPU the host list must have the GPU list's size
//   :955  allocFilterCoeffs, :964 uploadFilterCoeffsToGPU, :973 fdtd_start_simulation
//   :981-1025 fdtd_step per step, updateCurrentGridFromGPU
//   :909  fdtd_cleanup
//
// Build: compile this file with the reference's sources in place of
// simulator_dispatch.cpp, simulator_gpu.cpp, simulator_gpu.cu and
// sponge_kernel.cu, with -I<this repository>/include -I<this directory>,
// and link -L<repository>/virs_b200 -lvirs_b200.
//
// Errors: the reference prints CUDA errors and carries on, or exits
// (CUDA_CHECK, simulator_gpu.cu:11-19); here every failed library call
// throws std::runtime_error with virs_last_error()'s message.
//
// Ownership is the reference's: fdtd_setup allocates p_curr, p_next, p_prev,
// flags and normals (simulator_gpu.cpp:12-18), fdtd_start_simulation
// p_audio_output, allocFilterCoeffs biquad_coeffs, allocFilterStates
// biquad_state_ptr, and fdtd_cleanup frees them all and sets them to null
// (simulator_gpu.cpp:237-305), so ~VectorSpace deletes null pointers.  The
// binding frees only arrays it allocated itself (the reference frees
// whatever the Grid points to, uninitialised pointers included).
#include "simulator_dispatch.h"

#include <cstring>
#include <iostream>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include "virs.h"
#include "virs_dispatch.h"

namespace {

struct Binding {
    virs_sim *sim = nullptr;
    bool classified = false;       // virs_classify ran on the current flags
    bool fields_to_device = false; // updateGPUFromGrid asked for the host fields
    bool started = false;          // fdtd_start_simulation ran
    bool has_receiver = false;
    std::size_t rx = 334, ry = 225, rz = 270; // simulator_gpu.cu:295
    // host arrays this binding allocated (Grid's own members start
    // uninitialised, so only these are ever freed)
    float *p_curr = nullptr, *p_next = nullptr, *p_prev = nullptr;
    uint8_t *flags = nullptr, *normals = nullptr;
    float *audio = nullptr, *coeffs = nullptr, *states = nullptr;
};

std::mutex g_mu;
std::map<const VectorSpace *, Binding> g_bind;

Binding &of(VectorSpace *space)
{
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_bind.find(space);
    if (it == g_bind.end()) throw std::runtime_error("virs_dispatch: fdtd_setup was not called for this VectorSpace");
    return it->second;
}

void check(virs_status st, const char *what)
{
    if (st != VIRS_OK) throw std::runtime_error(std::string("virs_dispatch: ") + what + ": " + virs_last_error());
}

// the grid's flags, uploaded and classified (sponge, codes, normals,
// boundary list); the classified flags come back to the host as the
// reference's buildSpongeLayerGPU copies them back (sponge_kernel.cu:94-95)
void classify(VectorSpace *space, Binding &b)
{
    Grid &g = space->getGrid();
    check(virs_set_grid(b.sim, g.Nx, g.Ny, g.Nz, space->h, g.flags, nullptr), "virs_set_grid");
    check(virs_classify(b.sim), "virs_classify");
    check(virs_get_flags(b.sim, g.flags, g.size), "virs_get_flags");
    b.classified = true;
}

// free an array the binding allocated, and clear the Grid member that
// still points to it
template <typename T> void release(T *&mine, T *&member)
{
    if (member == mine) member = nullptr;
    delete[] mine;
    mine = nullptr;
}

} // namespace

void virs_dispatch_set_receiver(VectorSpace *space, std::size_t x, std::size_t y, std::size_t z)
{
    Binding &b = of(space);
    b.rx = x;
    b.ry = y;
    b.rz = z;
    b.has_receiver = true;
}

// simulator_dispatch.cpp:12-19 -> simulator_gpu.cpp:7-235
void fdtd_setup(VectorSpace *space)
{
    Grid &g = space->getGrid();
    virs_params p;
    check(virs_params_default(&p), "virs_params_default");
    p.cell_size = space->h;
    fdtd_cleanup(space); // a second set-up of the same VectorSpace starts over
    Binding b;
    check(virs_create(&p, &b.sim), "virs_create");
    g.p_curr = b.p_curr = new float[g.size]();
    g.p_next = b.p_next = new float[g.size]();
    g.p_prev = b.p_prev = new float[g.size]();
    g.flags = b.flags = new uint8_t[g.size]();
    g.normals = b.normals = new uint8_t[g.size]();
    g.p_source = space->audio_file.samples.empty() ? nullptr : space->audio_file.samples[0].data();
    g.allocated_filter_memory = false;
    std::lock_guard<std::mutex> lock(g_mu);
    g_bind[space] = b;
}

// simulator_dispatch.cpp:83-91 -> sponge_kernel.cu:65-99, and the normals,
// boundary list and filter states that loadObj builds next
// (simulator.cpp:480-610), all in virs_classify
void buildSpongeLayer(VectorSpace *space)
{
    classify(space, of(space));
}

// simulator_dispatch.cpp:70-81: the host flags and fields to the device.
// Flags that differ from the classified ones on the device (or were never
// classified) are uploaded and classified again; a classified grid keeps
// its flag-2 voxels, so classifying it again changes nothing.  The fields
// are uploaded once the simulation has started, because
// virs_start_simulation starts from rest.
void updateGPUFromGrid(VectorSpace *space)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    bool same = b.classified;
    if (same) {
        uint8_t *dev = new uint8_t[g.size];
        const virs_status st = virs_get_flags(b.sim, dev, g.size);
        same = st == VIRS_OK && std::memcmp(dev, g.flags, g.size) == 0;
        delete[] dev;
        check(st, "virs_get_flags");
    }
    if (!same) classify(space, b);
    b.fields_to_device = true;
    if (b.started) check(virs_set_pressure(b.sim, g.p_curr, g.p_prev, g.size), "virs_set_pressure");
}

// simulator_dispatch.cpp:102-109: the normals were computed from the
// classified flags by virs_classify (ENormals bits, normals.h:3-11).
void uploadNormalsToGPU(VectorSpace *space)
{
    of(space);
}

// simulator_dispatch.cpp:111-118: its body is commented out in the reference.
void uploadPZetaToGPU(VectorSpace *) {}

// simulator_dispatch.cpp:120-130: the GPU built the same ascending list of
// flag-2 voxels (simulator.cpp:572-605); the host list must have its size.
void uploadBoundaryIndicesToGPU(VectorSpace *space)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    virs_grid_info info;
    check(virs_get_grid_info(b.sim, &info), "virs_get_grid_info");
    if (info.boundary_count != g.boundary_indices_size)
        throw std::runtime_error("virs_dispatch: the host boundary list has " + std::to_string(g.boundary_indices_size) +
                                 " voxels, the classified grid " + std::to_string(info.boundary_count));
}

// simulator_dispatch.cpp:132-160: zeroed host states [nB][sections][4]; the
// device states are the handle's (zeroed by virs_set_filters and
// virs_start_simulation)
void allocFilterStates(VectorSpace *space)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    release(b.states, g.biquad_state_ptr);
    g.biquad_state_ptr = b.states = new float[g.num_filter_sections * g.boundary_indices_size * 4]();
    g.allocated_filter_memory = true;
}

// simulator_dispatch.cpp:162-250: zeroed host coefficients [materials][5]
void allocFilterCoeffs(VectorSpace *space, const size_t num_materials)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    g.num_materials = num_materials;
    release(b.coeffs, g.biquad_coeffs);
    g.biquad_coeffs = b.coeffs = new float[num_materials * 5]();
}

// simulator_dispatch.cpp:252-280: the reference's boundary kernel filters
// every boundary voxel with one section of coefficient set 0
// (simulator_gpu.cu:126-146); every wall voxel is absorber 0 here
// (virs_set_grid without wall materials), so set 0 is the one used.
void uploadFilterCoeffsToGPU(VectorSpace *space)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    check(virs_set_filters(b.sim, (uint32_t)g.num_materials, 1, g.biquad_coeffs), "virs_set_filters");
}

// simulator_dispatch.cpp:93-100: zeroed p_audio_output[steps]; receivers,
// the start from rest, and the host fields if updateGPUFromGrid sent them
void fdtd_start_simulation(VectorSpace *space, size_t steps)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    if (b.has_receiver || (b.rx < g.Nx && b.ry < g.Ny && b.rz < g.Nz)) {
        const uint64_t r = (uint64_t)g.idx(b.rx, b.ry, b.rz);
        check(virs_set_receivers(b.sim, 1, &r), "virs_set_receivers");
    } else {
        // the reference reads out of bounds here; its samples are undefined
        std::cerr << "virs_dispatch: the grid " << g.Nx << "x" << g.Ny << "x" << g.Nz
                  << " does not contain the receiver (334, 225, 270); recording zeros"
                     " (virs_dispatch_set_receiver names another voxel)"
                  << std::endl;
        check(virs_set_receivers(b.sim, 0, nullptr), "virs_set_receivers");
    }
    check(virs_start_simulation(b.sim, steps), "virs_start_simulation");
    b.started = true;
    if (b.fields_to_device) check(virs_set_pressure(b.sim, g.p_curr, g.p_prev, g.size), "virs_set_pressure");
    release(b.audio, g.p_audio_output);
    g.p_audio_output_size = steps;
    g.p_audio_output = b.audio = new float[steps]();
}

// simulator_dispatch.cpp:21-29 -> simulator_gpu.cu:184-332: one step, the
// receiver sample into p_audio_output[step], and the RMS stop rule
bool fdtd_step(VectorSpace *space, unsigned int step)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    int keep = 1;
    float v = 0.f;
    check(virs_step(b.sim, step, &keep, &v), "virs_step");
    if (step < g.p_audio_output_size) g.p_audio_output[step] = v;
    return keep != 0;
}

// simulator_dispatch.cpp:42-49
void updateCurrentGridFromGPU(VectorSpace *space)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    check(virs_get_pressure(b.sim, g.p_curr, nullptr, g.size), "virs_get_pressure");
}

// simulator_dispatch.cpp:31-40: p^n and p^{n-1}.  The reference's p_next
// then holds a stale buffer (p^{n-1}, simulator_gpu.cu:292-293); the library
// updates in place and keeps no third field, so p_next gets p^{n-1} too.
void updateAllGridFromGPU(VectorSpace *space)
{
    Binding &b = of(space);
    Grid &g = space->getGrid();
    check(virs_get_pressure(b.sim, g.p_curr, g.p_prev, g.size), "virs_get_pressure");
    std::memcpy(g.p_next, g.p_prev, g.size * sizeof(float));
}

// simulator_dispatch.cpp:60-68 -> init_sphere.cu:27-55
void initPressureSphere(VectorSpace *space, size_t xpos, size_t ypos, size_t zpos, size_t radius, float pressure,
                        bool init)
{
    Binding &b = of(space);
    check(virs_init_pressure_sphere(b.sim, xpos, ypos, zpos, radius, pressure, init ? 1 : 0),
          "virs_init_pressure_sphere");
}

// simulator_dispatch.cpp:51-58 -> simulator_gpu.cpp:237-305
void fdtd_cleanup(VectorSpace *space)
{
    Binding b;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        auto it = g_bind.find(space);
        if (it == g_bind.end()) return;
        b = it->second;
        g_bind.erase(it);
    }
    virs_destroy(b.sim);
    Grid &g = space->getGrid();
    release(b.p_curr, g.p_curr);
    release(b.p_next, g.p_next);
    release(b.p_prev, g.p_prev);
    release(b.flags, g.flags);
    release(b.normals, g.normals);
    release(b.audio, g.p_audio_output);
    release(b.coeffs, g.biquad_coeffs);
    release(b.states, g.biquad_state_ptr);
    g.p_source = nullptr;
    g.allocated_filter_memory = false;
}
