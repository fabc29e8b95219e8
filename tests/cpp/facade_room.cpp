// A C++ host of the library through include/virs.hpp: a 1.0 x 0.8 x 0.6 m
// shoebox (12 triangles, wall material 0) at 2.5 cm cells, one soft source
// and one receiver, the reference's default filter, N steps.  Prints the
// receiver samples, one per line (%.9g keeps every FP32 bit), or the
// library's error and its status as the exit code.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "virs.hpp"

int main(int argc, char **argv)
{
    const uint64_t steps = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 300;
    try {
        virs_params p = virs::default_params();
        p.cell_size = 0.025f;
        p.bbox_nudge = 0.f;
        virs::Simulator sim(p);
        const float X = 1.0f, Y = 0.8f, Z = 0.6f;
        const std::vector<float> v = {0, 0, 0, X, 0, 0, X, Y, 0, 0, Y, 0, 0, 0, Z, X, 0, Z, X, Y, Z, 0, Y, Z};
        const std::vector<uint32_t> t = {0, 1, 2, 0, 2, 3, 4, 6, 5, 4, 7, 6, 0, 4, 5, 0, 5, 1,
                                         1, 5, 6, 1, 6, 2, 2, 6, 7, 2, 7, 3, 3, 7, 4, 3, 4, 0};
        sim.set_mesh(v, t, std::vector<int32_t>(12, 0));
        sim.classify();
        const virs_grid_info g = sim.info();
        const auto at = [&](uint64_t x, uint64_t y, uint64_t z) { return (z * g.ny + y) * g.nx + x; };
        std::vector<float> sig(steps);
        for (uint64_t n = 0; n < steps; ++n) {
            const double u = ((double)n - 32.0) / 8.0;
            sig[n] = (float)(-u * std::exp(-0.5 * u * u));
        }
        sim.set_sources({at(g.nx / 2, g.ny / 2, g.nz / 2)}, sig);
        sim.set_receivers({at(g.nx / 4, g.ny / 3, g.nz / 2)});
        sim.start(steps);
        sim.run(steps);
        sim.synchronize();
        for (float s : sim.ir(0, steps, 1)) std::printf("%.9g\n", s);
    } catch (const virs::Error &e) {
        std::fprintf(stderr, "virs error %d: %s\n", (int)e.status, e.what());
        return 10 + (int)e.status;
    }
    return 0;
}
