// Filter coefficient design on the host.
//
//   rbj_highpass / rbj_lowpass   biquad.cpp:3-43, with the reference's
//                                float/double promotions (2.f * M_PI is a
//                                double, sin/cos of a float call the double
//                                functions, results narrowed to float);
//   virs_design_first_order,
//   virs_design_octave_cascade   FP64 bilinear-transform designs of
//                                absorbing-boundary filters (no reference
//                                counterpart); published formulas of the RBJ
//                                "Audio EQ Cookbook" for the shelves and the
//                                peaking section.
//
// Compiled with -ffp-contract=off.
#include <cmath>

#include "internal.hpp"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace virs {

void rbj_highpass(float fs, float cutoff, float q, float gain, float out5[5])
{
    const float omega = 2.f * M_PI * cutoff / fs;
    const float alpha = std::sin((double)omega) / (2.f * q);
    const float a0 = 1.f + alpha;
    float b0 = (1.f + std::cos((double)omega)) / 2.f / a0;
    float b1 = -(1.f + std::cos((double)omega)) / a0;
    float b2 = b0;
    const float a1 = -2.f * std::cos((double)omega) / a0;
    const float a2 = (1.f - alpha) / a0;
    b0 *= gain; b1 *= gain; b2 *= gain;
    out5[0] = b0; out5[1] = b1; out5[2] = b2; out5[3] = a1; out5[4] = a2;
}

void rbj_lowpass(float fs, float cutoff, float q, float gain, float out5[5])
{
    const float omega = 2.f * M_PI * cutoff / fs;
    const float alpha = std::sin((double)omega) / (2.f * q);
    const float a0 = 1.f + alpha;
    float b0 = (1.f - std::cos((double)omega)) / 2.f / a0;
    float b1 = (1.f - std::cos((double)omega)) / a0;
    float b2 = b0;
    const float a1 = -2.f * std::cos((double)omega) / a0;
    const float a2 = (1.f - alpha) / a0;
    b0 *= gain; b1 *= gain; b2 *= gain;
    out5[0] = b0; out5[1] = b1; out5[2] = b2; out5[3] = a1; out5[4] = a2;
}

// Sponge weight of a boundary voxel at squared distance d2 from the nearest
// wall: ((W + 1 - sqrt(d2)) / W)^2, computed in double, 1 at d2 = 1.
float sponge_weight(int W, int d2)
{
    double t = ((double)W + 1.0 - std::sqrt((double)d2)) / (double)W;
    if (t < 0.0) t = 0.0;
    return (float)(t * t);
}

} // namespace virs

extern "C" {

// First-order absorbing section: the bilinear transform (prewarped at fc) of
// H(s) = G * wc / (s + wc) with G = (1 - R) / (1 + R), R the pressure
// reflection coefficient.  b2 = a2 = 0.
__attribute__((visibility("default"))) virs_status virs_design_first_order(double fs, double reflection, double fc,
                                                                           double *out5)
{
    if (!out5 || !(fs > 0) || !(fc > 0) || !(fc < fs / 2) || !(reflection >= -1) || !(reflection < 1))
        return virs::fail(VIRS_E_ARG, "virs_design_first_order: need fs > 0, 0 < fc < fs/2, -1 <= R < 1");
    const double g = (1.0 - reflection) / (1.0 + reflection);
    const double k = std::tan(M_PI * fc / fs);
    out5[0] = g * k / (1.0 + k);
    out5[1] = g * k / (1.0 + k);
    out5[2] = 0.0;
    out5[3] = (k - 1.0) / (k + 1.0);
    out5[4] = 0.0;
    return VIRS_OK;
}

// Three-section absorbing cascade from octave-band absorption coefficients
// alpha[0..2] (low, mid, high): band gains G_b = (1 - R_b) / (1 + R_b) with
// R_b = sqrt(1 - alpha_b), realised as a low shelf at f[0] (gain G_0 below
// it, 1 above), a peaking section at f[1] (gain G_1 there, 1 far from it)
// and a high shelf at f[2] (gain G_2 above it).  RBJ cookbook formulas,
// shelf slope 1, peak Q = 1/sqrt(2); the cascade's gain is about G_b in band
// b.  freqs may be NULL for {250, 1000, 4000} Hz.  out15 = 3 x {b0 b1 b2 a1 a2}.
__attribute__((visibility("default"))) virs_status virs_design_octave_cascade(double fs, const double *alpha,
                                                                              const double *freqs, double *out15)
{
    if (!out15 || !alpha || !(fs > 0))
        return virs::fail(VIRS_E_ARG, "virs_design_octave_cascade: null argument or fs <= 0");
    const double f_def[3] = {250.0, 1000.0, 4000.0};
    const double *f = freqs ? freqs : f_def;
    double G[3];
    for (int b = 0; b < 3; ++b) {
        if (!(alpha[b] > 0.0) || !(alpha[b] <= 1.0))
            return virs::fail(VIRS_E_ARG, "virs_design_octave_cascade: absorption must be in (0, 1]");
        if (!(f[b] > 0.0) || !(f[b] < fs / 2))
            return virs::fail(VIRS_E_ARG, "virs_design_octave_cascade: band frequency outside (0, fs/2)");
        const double R = std::sqrt(1.0 - alpha[b]);
        G[b] = (1.0 - R) / (1.0 + R);
    }
    auto norm = [](double *o, double b0, double b1, double b2, double a0, double a1, double a2) {
        o[0] = b0 / a0; o[1] = b1 / a0; o[2] = b2 / a0; o[3] = a1 / a0; o[4] = a2 / a0;
    };
    // low shelf carrying G[0] below f[0] relative to 1 above, then scaled
    // so that the section passes G[0] at DC and 1 at high frequencies
    {
        const double A = std::sqrt(G[0]);
        const double w = 2.0 * M_PI * f[0] / fs, cw = std::cos(w), al = std::sin(w) / 2.0 * std::sqrt(2.0);
        const double sA = 2.0 * std::sqrt(A) * al;
        norm(out15, A * ((A + 1) - (A - 1) * cw + sA), 2 * A * ((A - 1) - (A + 1) * cw), A * ((A + 1) - (A - 1) * cw - sA),
             (A + 1) + (A - 1) * cw + sA, -2 * ((A - 1) + (A + 1) * cw), (A + 1) + (A - 1) * cw - sA);
    }
    // peaking section around f[1] with gain G[1] (relative to 1)
    {
        const double A = std::sqrt(G[1]);
        const double w = 2.0 * M_PI * f[1] / fs, cw = std::cos(w), al = std::sin(w) / (2.0 / std::sqrt(2.0));
        norm(out15 + 5, 1 + al * A, -2 * cw, 1 - al * A, 1 + al / A, -2 * cw, 1 - al / A);
    }
    // high shelf with gain G[2] above f[2]
    {
        const double A = std::sqrt(G[2]);
        const double w = 2.0 * M_PI * f[2] / fs, cw = std::cos(w), al = std::sin(w) / 2.0 * std::sqrt(2.0);
        const double sA = 2.0 * std::sqrt(A) * al;
        norm(out15 + 10, A * ((A + 1) + (A - 1) * cw + sA), -2 * A * ((A - 1) + (A + 1) * cw),
             A * ((A + 1) + (A - 1) * cw - sA), (A + 1) - (A - 1) * cw + sA, 2 * ((A - 1) - (A + 1) * cw),
             (A + 1) - (A - 1) * cw - sA);
    }
    return VIRS_OK;
}

} // extern "C"
