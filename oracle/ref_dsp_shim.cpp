// Harness around the reference's anti-alias filter code (TEST
// INFRASTRUCTURE), compiled from the reference tree as it is:
// src/util/downsampling_filter_iir.cpp (designChebyshevI_LP :58-193 with
// distributeDCGain :11-56, initState / processBlock :197-240).  C linkage
// for ctypes.
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "downsampling_filter_iir.h"

extern "C" {

// sos out [max][6] {b0, b1, b2, a0, a1, a2}; returns the section count, or
// -1 when the design throws, -2 when max is too small
__attribute__((visibility("default"))) int ref_cheby_design(double fs, double fc, double fstop, double ap_db,
                                                             double as_db, double *out, int max)
{
    std::vector<Biquad> sos;
    try {
        sos = designChebyshevI_LP(fs, fc, fstop, ap_db, as_db);
    } catch (const std::exception &) {
        return -1;
    }
    if ((int)sos.size() > max) return -2;
    for (size_t i = 0; i < sos.size(); ++i) {
        const Biquad &b = sos[i];
        const double v[6] = {b.b0, b.b1, b.b2, b.a0, b.a1, b.a2};
        for (int j = 0; j < 6; ++j) out[6 * i + j] = v[j];
    }
    return (int)sos.size();
}

// one channel through the cascade from a zero state
__attribute__((visibility("default"))) void ref_cheby_process(const double *sos6, int n, const float *in, float *out,
                                                              uint64_t frames)
{
    std::vector<Biquad> sos((size_t)n);
    for (int i = 0; i < n; ++i)
        sos[(size_t)i] = Biquad{sos6[6 * i], sos6[6 * i + 1], sos6[6 * i + 2], sos6[6 * i + 3], sos6[6 * i + 4],
                                sos6[6 * i + 5]};
    IIRState st;
    initState(st, sos, 1);
    processBlock(sos, st, in, out, (std::size_t)frames);
}

} // extern "C"
