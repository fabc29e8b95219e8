// Test stand-in for src/simulator/simulator_dispatch.h of the Snipet/VIRS
// tree: the dispatch functions with the signatures declared at
// simulator_dispatch.h:4-25.
#pragma once

#include <cstddef>

#include "vectorspace.h"

void fdtd_setup(VectorSpace *space);
bool fdtd_step(VectorSpace *space, unsigned int step);
void fdtd_cleanup(VectorSpace *space);
void fdtd_start_simulation(VectorSpace *space, std::size_t steps);
void initPressureSphere(VectorSpace *space, std::size_t xpos, std::size_t ypos, std::size_t zpos, std::size_t radius,
                        float pressure, bool init);
void buildSpongeLayer(VectorSpace *space);
void updateAllGridFromGPU(VectorSpace *space);
void updateCurrentGridFromGPU(VectorSpace *space);
void updateGPUFromGrid(VectorSpace *space);
void uploadNormalsToGPU(VectorSpace *space);
void uploadPZetaToGPU(VectorSpace *space);
void uploadBoundaryIndicesToGPU(VectorSpace *space);
void allocFilterStates(VectorSpace *space);
void allocFilterCoeffs(VectorSpace *space, const std::size_t num_materials);
void uploadFilterCoeffsToGPU(VectorSpace *space);
