/* virs.hpp -- C++ facade over the C ABI of virs.h.
 *
 * The reference drives its GPU step through the class `Simulator`
 * (src/simulator/simulator.h:19-86): loadObj, then simulate (N steps),
 * then the impulse response.  `virs::Simulator` gives a C++ host the same
 * flow over libvirs_b200, with RAII ownership of the handle and exceptions
 * instead of status codes.  Header-only: link with -lvirs_b200. */
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "virs.h"

namespace virs {

/* a failed call: the status and virs_last_error() of the calling thread */
class Error : public std::runtime_error {
public:
    Error(virs_status s, const char *what) : std::runtime_error(what ? what : "virs error"), status(s) {}
    virs_status status;
};

inline void check(virs_status s)
{
    if (s != VIRS_OK) throw Error(s, virs_last_error());
}

inline virs_params default_params()
{
    virs_params p;
    check(virs_params_default(&p));
    return p;
}

class Simulator {
public:
    explicit Simulator(const virs_params &p = default_params()) { check(virs_create(&p, &h_)); }
    ~Simulator()
    {
        if (h_) virs_destroy(h_);
    }
    Simulator(const Simulator &) = delete;
    Simulator &operator=(const Simulator &) = delete;
    Simulator(Simulator &&o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
    Simulator &operator=(Simulator &&o) noexcept
    {
        if (this != &o) {
            if (h_) virs_destroy(h_);
            h_ = std::exchange(o.h_, nullptr);
        }
        return *this;
    }

    virs_sim *handle() const { return h_; }

    /* geometry: Simulator::loadObj (simulator.cpp:262-452) */
    void set_material_roles(const std::vector<uint8_t> &roles)
    {
        check(virs_set_material_roles(h_, roles.data(), roles.size()));
    }
    void load_obj(const std::string &path) { check(virs_load_obj(h_, path.c_str())); }
    void set_mesh(const std::vector<float> &verts, const std::vector<uint32_t> &tris,
                  const std::vector<int32_t> &tri_material)
    {
        check(virs_set_mesh(h_, verts.data(), verts.size() / 3, tris.data(), tri_material.data(), tris.size() / 3));
    }
    /* one z-slab of a grid split over several GPUs: slab `part` of `parts`
     * from a mesh, or owned planes [z_lo, z_hi) from the whole grid's flags
     * (planes [z_first, z_first + flags.size()/(nx*ny))) */
    void set_mesh_slab(const std::vector<float> &verts, const std::vector<uint32_t> &tris,
                       const std::vector<int32_t> &tri_material, uint32_t part, uint32_t parts)
    {
        check(virs_set_mesh_slab(h_, verts.data(), verts.size() / 3, tris.data(), tri_material.data(),
                                 tris.size() / 3, part, parts));
    }
    void load_obj_slab(const std::string &path, uint32_t part, uint32_t parts)
    {
        check(virs_load_obj_slab(h_, path.c_str(), part, parts));
    }
    void set_grid_slab(uint64_t nx, uint64_t ny, uint64_t nz, float cell_size, uint64_t z_lo, uint64_t z_hi,
                       const std::vector<uint8_t> &flags, const std::vector<uint8_t> &wall_material, uint64_t z_first)
    {
        check(virs_set_grid_slab(h_, nx, ny, nz, cell_size, z_lo, z_hi, flags.data(),
                                 wall_material.empty() ? nullptr : wall_material.data(), z_first,
                                 flags.size() / (nx * ny)));
    }
    struct SlabPlanes {
        void *first, *last, *ghost_lo, *ghost_hi;
        size_t bytes;
    };
    /* the planes of p^n to exchange before the next step */
    SlabPlanes slab_planes() const
    {
        SlabPlanes p{};
        check(virs_slab_planes(h_, &p.first, &p.last, &p.ghost_lo, &p.ghost_hi, &p.bytes));
        return p;
    }
    /* sponge layer, normals, boundary list: the rest of loadObj (:469-610) */
    void classify() { check(virs_classify(h_)); }
    virs_grid_info info() const
    {
        virs_grid_info g;
        check(virs_get_grid_info(h_, &g));
        return g;
    }
    uint64_t voxels() const
    {
        const virs_grid_info g = info();
        return g.nx * g.ny * g.nz;
    }
    std::vector<uint8_t> flags() const
    {
        std::vector<uint8_t> f(voxels());
        check(virs_get_flags(h_, f.data(), f.size()));
        return f;
    }
    std::vector<uint8_t> wall_materials() const
    {
        std::vector<uint8_t> w(voxels());
        check(virs_get_wall_materials(h_, w.data(), w.size()));
        return w;
    }
    std::vector<uint32_t> boundary_indices() const
    {
        std::vector<uint32_t> b(info().boundary_count);
        check(virs_get_boundary_indices(h_, b.data(), b.size()));
        return b;
    }

    /* filters: coeffs [n_materials][n_sections][5] {b0, b1, b2, a1, a2} */
    void set_filters(uint32_t n_materials, uint32_t n_sections, const std::vector<float> &coeffs)
    {
        check(virs_set_filters(h_, n_materials, n_sections, coeffs.data()));
    }
    /* soft sources: signal [n][len]; receivers by voxel index */
    void set_sources(const std::vector<uint64_t> &idx, const std::vector<float> &signal)
    {
        check(virs_set_sources(h_, (uint32_t)idx.size(), idx.data(), signal.data(),
                               idx.empty() ? 0 : signal.size() / idx.size()));
    }
    void set_receivers(const std::vector<uint64_t> &idx)
    {
        check(virs_set_receivers(h_, (uint32_t)idx.size(), idx.data()));
    }

    /* Simulator::simulate (simulator.cpp:933-1025): start from rest, run */
    void start(uint64_t steps) { check(virs_start_simulation(h_, steps)); }
    void run(uint64_t steps, void *stream = nullptr) { check(virs_run(h_, steps, stream)); }
    void synchronize() { check(virs_synchronize(h_)); }
    /* right after start: the fastest tiling and steps per pass for this grid */
    virs_tiling autotune(uint32_t trial_steps = 4)
    {
        virs_tiling t{};
        check(virs_autotune(h_, trial_steps, &t));
        return t;
    }
    /* two steps per pass over the fields (bit-identical to single steps) */
    void set_time_blocking(int steps_per_pass, int tile_rows = 0, int planes_per_block = 0)
    {
        check(virs_set_time_blocking(h_, steps_per_pass, tile_rows, planes_per_block));
    }
    /* receiver samples [n_receivers][steps] from step `first` */
    std::vector<float> ir(uint64_t first, uint64_t steps, uint32_t n_receivers) const
    {
        std::vector<float> out((size_t)n_receivers * steps);
        check(virs_get_ir(h_, first, steps, out.data()));
        return out;
    }
    std::vector<float> pressure() const
    {
        std::vector<float> p(voxels());
        check(virs_get_pressure(h_, p.data(), nullptr, p.size()));
        return p;
    }

private:
    virs_sim *h_ = nullptr;
};

} // namespace virs
