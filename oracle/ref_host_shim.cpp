// Harness around reference host code compiled from the reference tree
// (TEST INFRASTRUCTURE).  It exposes, with C linkage:
//   - triangleBoxOverlap3  (src/simulator/simulator.cpp:45-141, cut out by
//     oracle/Makefile into _ref/sat_extract.inc together with the Vec3f
//     struct of src/simulator/vectorspace.h:12-44 and the vector helpers of
//     simulator.cpp:22-43);
//   - computeHighpassBiquad / computeLowpassBiquad (src/simulator/biquad.cpp,
//     linked as it is).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <initializer_list>

#include "sat_extract.inc"
#include "biquad.h"

extern "C" {

__attribute__((visibility("default"))) int ref_sat(const float *a, const float *b, const float *c,
                                                    const float *lo, const float *hi)
{
    return triangleBoxOverlap3(Vec3f(a[0], a[1], a[2]), Vec3f(b[0], b[1], b[2]), Vec3f(c[0], c[1], c[2]),
                               Vec3f(lo[0], lo[1], lo[2]), Vec3f(hi[0], hi[1], hi[2]))
               ? 1
               : 0;
}

// Many SAT queries in one call: tris [n][9], boxes [n][6] (min xyz, max xyz).
__attribute__((visibility("default"))) void ref_sat_batch(const float *tris, const float *boxes, uint64_t n,
                                                          uint8_t *out)
{
    for (uint64_t i = 0; i < n; ++i) {
        const float *t = tris + 9 * i, *b = boxes + 6 * i;
        out[i] = (uint8_t)ref_sat(t, t + 3, t + 6, b, b + 3);
    }
}

__attribute__((visibility("default"))) void ref_highpass(float fs, float fc, float q, float g, float *out5)
{
    BiquadCoeffs k = computeHighpassBiquad(fs, fc, q, g);
    out5[0] = k.b0; out5[1] = k.b1; out5[2] = k.b2; out5[3] = k.a1; out5[4] = k.a2;
}

__attribute__((visibility("default"))) void ref_lowpass(float fs, float fc, float q, float g, float *out5)
{
    BiquadCoeffs k = computeLowpassBiquad(fs, fc, q, g);
    out5[0] = k.b0; out5[1] = k.b1; out5[2] = k.b2; out5[3] = k.a1; out5[4] = k.a2;
}

} // extern "C"
