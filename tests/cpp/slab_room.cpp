// A C++ host of the C ABI that splits one grid into z-slabs: a 1.2 x 1.0 x
// 0.9 m room with two boxes inside (two absorbing materials, 3-section
// cascades), sponge width 4, one soft source and three receivers at
// different heights.  The whole grid runs on one handle; the same grid runs
// as `parts` slab handles (virs_set_mesh_slab: each voxelises only its
// planes) advanced by virs_slab_run, which exchanges the ghost planes before
// every step.  Every receiver sample and the p^n and p^{n-1} of every owned
// plane must equal the whole grid's bit for bit.
//
//   slab_room <parts> <steps> <storage 0|1|2>      exit 0: equal
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "virs.h"

namespace {

struct Mesh {
    std::vector<float> v;
    std::vector<uint32_t> t;
    std::vector<int32_t> m;
    void box(float x0, float y0, float z0, float x1, float y1, float z1, int32_t mat)
    {
        const uint32_t b = (uint32_t)(v.size() / 3);
        const float c[8][3] = {{x0, y0, z0}, {x1, y0, z0}, {x0, y1, z0}, {x1, y1, z0},
                               {x0, y0, z1}, {x1, y0, z1}, {x0, y1, z1}, {x1, y1, z1}};
        for (auto &p : c) v.insert(v.end(), p, p + 3);
        const uint32_t q[6][4] = {{0, 2, 6, 4}, {1, 5, 7, 3}, {0, 4, 5, 1}, {2, 3, 7, 6}, {0, 1, 3, 2}, {4, 6, 7, 5}};
        for (auto &f : q) {
            const uint32_t tri[6] = {f[0], f[1], f[2], f[0], f[2], f[3]};
            for (uint32_t k : tri) t.push_back(b + k);
            m.push_back(mat);
            m.push_back(mat);
        }
    }
};

int fails = 0;
void check(virs_status st, const char *what)
{
    if (st != VIRS_OK) {
        std::fprintf(stderr, "%s: status %d: %s\n", what, (int)st, virs_last_error());
        std::exit(10 + (int)st);
    }
}

// a configured handle: whole grid (parts == 0) or slab `part` of `parts`
virs_sim *make(const Mesh &mesh, int storage, uint32_t part, uint32_t parts)
{
    virs_params p;
    check(virs_params_default(&p), "params");
    p.cell_size = 0.025f;
    p.bbox_nudge = 0.f;
    p.sponge_width = 4;
    p.storage = storage;
    p.storage_scale = storage ? 1024.f : 0.f;
    virs_sim *s = nullptr;
    check(virs_create(&p, &s), "create");
    const uint8_t roles[2] = {0, 1};
    check(virs_set_material_roles(s, roles, 2), "roles");
    if (parts == 0)
        check(virs_set_mesh(s, mesh.v.data(), mesh.v.size() / 3, mesh.t.data(), mesh.m.data(), mesh.m.size()), "mesh");
    else
        check(virs_set_mesh_slab(s, mesh.v.data(), mesh.v.size() / 3, mesh.t.data(), mesh.m.data(), mesh.m.size(),
                                 part, parts),
              "mesh slab");
    check(virs_classify(s), "classify");
    virs_grid_info g;
    check(virs_get_grid_info(s, &g), "info");
    const double alpha[2][3] = {{0.2, 0.4, 0.6}, {0.5, 0.3, 0.1}};
    std::vector<float> coef;
    for (auto &a : alpha) {
        double c[15];
        check(virs_design_octave_cascade(g.sample_rate, a, nullptr, c), "design");
        for (double x : c) coef.push_back((float)x);
    }
    check(virs_set_filters(s, 2, 3, coef.data()), "filters");
    return s;
}

} // namespace

int main(int argc, char **argv)
{
    const uint32_t parts = argc > 1 ? (uint32_t)std::atoi(argv[1]) : 3;
    const uint64_t steps = argc > 2 ? std::strtoull(argv[2], nullptr, 10) : 200;
    const int storage = argc > 3 ? std::atoi(argv[3]) : 0;
    Mesh mesh;
    mesh.box(0.f, 0.f, 0.f, 1.2f, 1.0f, 0.9f, 0);
    mesh.box(0.2f, 0.15f, 0.f, 0.5f, 0.45f, 0.4f, 1);
    mesh.box(0.7f, 0.5f, 0.3f, 1.0f, 0.8f, 0.6f, 1);

    virs_sim *whole = make(mesh, storage, 0, 0);
    virs_grid_info g;
    check(virs_get_grid_info(whole, &g), "info");
    const uint64_t nx = g.nx, ny = g.ny, nz = g.nz, plane = nx * ny;
    const auto at = [&](uint64_t x, uint64_t y, uint64_t z) { return (z * ny + y) * nx + x; };
    const uint64_t src = at(nx / 2, ny / 3, nz / 2);
    const uint64_t rcv[3] = {at(nx / 3, ny / 2, 3), at(2 * nx / 3, ny / 4, nz / 2 + 1), at(nx / 4, 2 * ny / 3, nz - 4)};
    std::vector<float> sig(steps);
    for (uint64_t n = 0; n < steps; ++n) {
        const double u = ((double)n - 24.0) / 6.0;
        sig[n] = (float)(-u * std::exp(-0.5 * u * u));
    }
    check(virs_set_sources(whole, 1, &src, sig.data(), steps), "sources");
    check(virs_set_receivers(whole, 3, rcv), "receivers");
    check(virs_start_simulation(whole, steps), "start");
    check(virs_run(whole, steps, nullptr), "run");
    std::vector<float> want_ir(3 * steps), want_p(plane * nz), want_q(plane * nz);
    check(virs_get_ir(whole, 0, steps, want_ir.data()), "ir");
    check(virs_get_pressure(whole, want_p.data(), want_q.data(), want_p.size()), "pressure");

    std::vector<virs_sim *> slab(parts);
    std::vector<uint64_t> lo(parts), hi(parts);
    std::vector<std::vector<int>> owned(parts);
    for (uint32_t k = 0; k < parts; ++k) {
        slab[k] = make(mesh, storage, k, parts);
        uint64_t gnz = 0;
        check(virs_get_slab_info(slab[k], &lo[k], &hi[k], &gnz), "slab info");
        if (gnz != nz) return 2;
        const uint64_t off = (lo[k] - 1) * plane;
        const uint64_t z_src = src / plane;
        if (z_src >= lo[k] && z_src < hi[k]) {
            const uint64_t l = src - off;
            check(virs_set_sources(slab[k], 1, &l, sig.data(), steps), "slab sources");
        }
        std::vector<uint64_t> loc;
        for (int r = 0; r < 3; ++r)
            if (rcv[r] / plane >= lo[k] && rcv[r] / plane < hi[k]) {
                loc.push_back(rcv[r] - off);
                owned[k].push_back(r);
            }
        check(virs_set_receivers(slab[k], (uint32_t)loc.size(), loc.data()), "slab receivers");
        check(virs_start_simulation(slab[k], steps), "slab start");
    }
    check(virs_slab_run(slab.data(), parts, steps), "slab run");
    for (uint32_t k = 0; k < parts; ++k) {
        check(virs_synchronize(slab[k]), "synchronize");
        const uint64_t nzl = hi[k] - lo[k] + 2;
        std::vector<float> ir(owned[k].size() * steps), p(plane * nzl), q(plane * nzl);
        if (!owned[k].empty()) check(virs_get_ir(slab[k], 0, steps, ir.data()), "slab ir");
        for (size_t j = 0; j < owned[k].size(); ++j)
            if (std::memcmp(&ir[j * steps], &want_ir[(size_t)owned[k][j] * steps], steps * sizeof(float)) != 0) {
                std::fprintf(stderr, "slab %u: receiver %d differs\n", k, owned[k][j]);
                ++fails;
            }
        check(virs_get_pressure(slab[k], p.data(), q.data(), p.size()), "slab pressure");
        const size_t bytes = (hi[k] - lo[k]) * plane * sizeof(float);
        if (std::memcmp(&p[plane], &want_p[lo[k] * plane], bytes) != 0 ||
            std::memcmp(&q[plane], &want_q[lo[k] * plane], bytes) != 0) {
            std::fprintf(stderr, "slab %u: fields of planes %llu..%llu differ\n", k, (unsigned long long)lo[k],
                         (unsigned long long)hi[k] - 1);
            ++fails;
        }
        virs_destroy(slab[k]);
    }
    float peak = 0.f;
    for (float x : want_ir) peak = std::fmax(peak, std::fabs(x));
    virs_destroy(whole);
    std::printf("%u slabs, %llu steps, storage %d, grid %llux%llux%llu, receiver peak %g: %s\n", parts,
                (unsigned long long)steps, storage, (unsigned long long)nx, (unsigned long long)ny,
                (unsigned long long)nz, peak, fails ? "DIFFERENT" : "equal");
    return fails || !(peak > 0.f) ? 1 : 0;
}
