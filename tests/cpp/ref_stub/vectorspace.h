// Test stand-in for src/simulator/vectorspace.h of the Snipet/VIRS tree:
// struct Grid with the members of vectorspace.h:46-105 that the dispatch
// layer uses, under the same names and types, and a VectorSpace with the
// constructor signature, getGrid() and h of vectorspace.h:176-231.  Like the
// reference's constructor (vectorspace.cpp:8-34), it only records the sizes:
// fdtd_setup allocates the host arrays.
#pragma once

#include <cstddef>
#include <cstdint>

#include "AudioFile.h"

struct Grid {
    float *p_curr, *p_next, *p_prev, *p_temp;
    uint8_t *flags;
    float *p_source;
    uint8_t *normals;
    std::size_t num_materials;
    float *biquad_coeffs;
    std::size_t num_filter_sections;
    float *biquad_state_ptr;
    bool allocated_filter_memory;
    uint32_t *boundary_indices;
    std::size_t boundary_indices_size;
    std::size_t Nx, Ny, Nz, size;
    std::size_t p_source_size;
    float *p_audio_output;
    std::size_t p_audio_output_size;
    float percent_to_target_RMS = 0.f;
    float rms_filter_state;

    inline std::size_t idx(std::size_t x, std::size_t y, std::size_t z) { return z * Ny * Nx + y * Nx + x; }
};

class VectorSpace {
public:
    VectorSpace(std::size_t x, std::size_t y, std::size_t z, const AudioFile<float> &audio, float h) : h(h)
    {
        grid.Nx = x;
        grid.Ny = y;
        grid.Nz = z;
        grid.size = x * y * z;
        grid.p_source_size = audio.getNumSamplesPerChannel();
        audio_file = audio;
    }
    ~VectorSpace()
    {
        delete[] grid.p_curr;
        delete[] grid.p_next;
        delete[] grid.flags;
    }
    Grid &getGrid() { return grid; }

    float h;
    AudioFile<float> audio_file;

private:
    Grid grid{};
};
