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
//                                peaking section;
//   virs_design_chebyshev_lowpass
//                                the anti-alias low-pass of the IR
//                                post-processing: designChebyshevI_LP and
//                                distributeDCGain
//                                (src/util/downsampling_filter_iir.cpp:11-193),
//                                the same steps and precisions (FP64, the DC
//                                gain in long double), so the sections are
//                                the reference's bit for bit.
//
// Compiled with -ffp-contract=off.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

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


// Chebyshev-I low-pass, second-order sections {b0, b1, b2, a0, a1, a2}:
// prewarped analogue edges, the order that meets the ripple and
// attenuation specs, the analogue poles ordered by imaginary part and
// taken two at a time (the first of each two with its conjugate makes a
// section with a double zero at z = -1; a last single pole makes a
// first-order section), bilinear transform, and the DC gain set to 1 by
// one common factor per section plus a final correction of section 0.
__attribute__((visibility("default"))) virs_status virs_design_chebyshev_lowpass(double fs, double fc, double fstop,
                                                                                 double ripple_db, double atten_db,
                                                                                 double *sos, uint32_t max_sections,
                                                                                 uint32_t *n_sections)
{
    if (!sos || !n_sections) return virs::fail(VIRS_E_ARG, "virs_design_chebyshev_lowpass: null argument");
    if (!(fs > 0) || !(fc > 0) || !(fc < 0.5 * fs))
        return virs::fail(VIRS_E_ARG, "virs_design_chebyshev_lowpass: need fs > 0 and 0 < fc < fs/2");
    if (fstop <= 0.0) fstop = std::min(0.499 * fs, 1.15 * fc);
    if (!(fstop > fc)) return virs::fail(VIRS_E_ARG, "virs_design_chebyshev_lowpass: the stop edge must lie above fc");
    const auto acosh_ = [](double x) { return std::log(x + std::sqrt(x * x - 1.0)); };
    const auto asinh_ = [](double x) { return std::log(x + std::sqrt(x * x + 1.0)); };
    const double T = 1.0 / fs, W = 2.0 / T;
    const double wp = 2.0 / T * std::tan(M_PI * (fc / fs));
    const double ws = 2.0 / T * std::tan(M_PI * (fstop / fs));
    const double eps = std::sqrt(std::pow(10.0, ripple_db / 10.0) - 1.0);
    const double order =
        acosh_(std::sqrt((std::pow(10.0, atten_db / 10.0) - 1.0) / (std::pow(10.0, ripple_db / 10.0) - 1.0))) /
        acosh_(ws / wp);
    const int N = std::max(1, (int)std::ceil(order));
    const double a = asinh_(1.0 / eps) / N;
    std::vector<std::complex<double>> poles;
    for (int k = 1; k <= N; ++k) {
        const double th = M_PI * (2.0 * k - 1.0) / (2.0 * N);
        std::complex<double> p(-std::sinh(a) * std::sin(th) * wp, std::cosh(a) * std::cos(th) * wp);
        if (p.real() >= 0) p = {-std::fabs(p.real()), p.imag()};
        poles.push_back(p);
    }
    std::sort(poles.begin(), poles.end(), [](const auto &x, const auto &y) { return x.imag() < y.imag(); });
    std::vector<double> o;
    for (int i = 0; i < N;) {
        const std::complex<double> p = poles[(size_t)i];
        double b[3], d[3];
        if (i + 1 == N || std::fabs(p.imag()) < 1e-12) {
            b[0] = 1.0; b[1] = 1.0; b[2] = 0.0;
            d[0] = W - p.real(); d[1] = -(W + p.real()); d[2] = 0.0;
            ++i;
        } else {
            const double m2 = p.real() * p.real() + p.imag() * p.imag();
            b[0] = 1.0; b[1] = 2.0; b[2] = 1.0;
            d[0] = W * W - 2.0 * p.real() * W + m2;
            d[1] = 2.0 * (m2 - W * W);
            d[2] = W * W + 2.0 * p.real() * W + m2;
            i += 2;
        }
        const double inv = 1.0 / d[0];
        o.insert(o.end(), {b[0] * inv, b[1] * inv, b[2] * inv, 1.0, d[1] * inv, d[2] * inv});
    }
    const size_t n = o.size() / 6;
    if (n > max_sections) return virs::fail(VIRS_E_ARG, "virs_design_chebyshev_lowpass: needs " + std::to_string(n) +
                                                            " sections, room for " + std::to_string(max_sections));
    const auto dc = [&]() {
        long double h = 1.0L;
        for (size_t q = 0; q < n; ++q) {
            const double *s = &o[6 * q];
            h *= ((long double)s[0] + s[1] + s[2]) / ((long double)s[3] + s[4] + s[5]);
        }
        return h;
    };
    const long double h = dc();
    if (std::isfinite((double)h) && fabsl(h) >= 1e-300L) {
        const long double g = powl(1.0L / h, 1.0L / (long double)n);
        for (size_t q = 0; q < n; ++q)
            for (int j = 0; j < 3; ++j) o[6 * q + j] = (double)((long double)o[6 * q + j] * g);
        const long double c = 1.0L / dc();
        for (int j = 0; j < 3; ++j) o[j] = (double)((long double)o[j] * c);
    }
    std::copy(o.begin(), o.end(), sos);
    *n_sections = (uint32_t)n;
    return VIRS_OK;
}

} // extern "C"
