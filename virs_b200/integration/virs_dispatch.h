// virs_dispatch.h -- what the libvirs_b200 binding of the reference's dispatch
// layer adds to src/simulator/simulator_dispatch.h.
//
// virs_dispatch.cpp implements every function of simulator_dispatch.h:4-25
// over the C ABI of virs.h.  The reference records the fixed voxel
// (334, 225, 270) (simulator_gpu.cu:295-300) and reads out of bounds on grids
// that do not contain it; the binding records that voxel when the grid
// contains it, and otherwise the voxel named here.
#pragma once

#include <cstddef>

class VectorSpace;

// The voxel whose pressure fdtd_step writes to p_audio_output[step]; call
// after fdtd_setup and before fdtd_start_simulation.
void virs_dispatch_set_receiver(VectorSpace *space, std::size_t x, std::size_t y, std::size_t z);
