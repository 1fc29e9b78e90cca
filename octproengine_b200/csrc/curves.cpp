// Curve generators of the OCT chain: the resampling (k-linearisation) curve,
// the dispersion phase and the spectral window, evaluated with the same float
// operations in the same order as the reference ProcessorConfiguration
// (src/core/processorconfiguration.cpp:438-589), so the tables handed to the
// kernels are bit-identical to what the reference backends receive. This file
// must be compiled without FP contraction (-ffp-contract=off) and without
// fast-math; on x86-64 float arithmetic is then IEEE single precision.
#include <cmath>
#include <cstddef>
#include <cstdint>

#include "../../include/ope_b200.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

float clampf(float v, float lo, float hi) { return (v < lo) ? lo : ((v > hi) ? hi : v); }

}  // namespace

extern "C" {

// r(i) = c0 + i*(c1' + i*(c2' + i*c3')), c_k' = c_k / (n-1)^k, clamped to
// [7, n-9] (processorconfiguration.cpp:438-459).
int ope_b200_generate_resampling_curve(int32_t n, const float coeffs[4], float* out) {
    if (n <= 0 || !coeffs || !out) return OPE_B200_E_INVALID;
    const float s1 = static_cast<float>(static_cast<size_t>(n)) - 1.0f;
    const float c0 = coeffs[0];
    const float c1 = coeffs[1] / s1;
    const float c2 = coeffs[2] / (s1 * s1);
    const float c3 = coeffs[3] / (s1 * s1 * s1);
    const float lo = 7.0f;
    const float hi = static_cast<float>(static_cast<size_t>(n) - 9);
    for (int32_t i = 0; i < n; ++i) {
        const float x = static_cast<float>(i);
        const float v = c0 + x * (c1 + x * (c2 + x * c3));
        out[i] = clampf(v, lo, hi);
    }
    return OPE_B200_OK;
}

// phase(i) = d0 + i*(d1' + i*(d2' + i*d3')), d_k' = d_k/(n-1)^k
// (processorconfiguration.cpp:461-482). The reference never applies `factor`.
int ope_b200_generate_dispersion_phase(int32_t n, const float coeffs[4], float* out) {
    if (n <= 0 || !coeffs || !out) return OPE_B200_E_INVALID;
    const float den = static_cast<float>(static_cast<size_t>(n) - 1);
    const float d0 = coeffs[0];
    const float d1 = coeffs[1] / den;
    const float d2 = coeffs[2] / (den * den);
    const float d3 = coeffs[3] / (den * den * den);
    for (int32_t i = 0; i < n; ++i) {
        const float x = static_cast<float>(static_cast<size_t>(i));
        out[i] = d0 + x * (d1 + x * (d2 + x * d3));
    }
    return OPE_B200_OK;
}

// Window types follow ope::WindowType (HANN, GAUSS, SINE, LANCZOS, RECTANGULAR,
// FLAT_TOP); shapes and the zeroed tails follow processorconfiguration.cpp:484-589.
int ope_b200_generate_window_curve(int32_t n, int32_t type, float center, float fill, float* out) {
    if (n <= 0 || !out || type < 0 || type > 5) return OPE_B200_E_INVALID;
    const unsigned size = static_cast<unsigned>(n);
    float cpos = center;
    if (cpos > 1.0f) cpos = 1.0f;
    if (cpos < 0.0f) cpos = 0.0f;
    const unsigned width = static_cast<unsigned>(fill * static_cast<float>(size));
    const unsigned ctr = static_cast<unsigned>(cpos * static_cast<float>(size));
    const int min_pos = static_cast<int>(ctr - width / 2);
    const float wm1 = static_cast<float>(width) - 1.0f;
    for (unsigned i = 0; i < size; ++i) {
        if (type == 1) {  // GAUSS
            const int xi = static_cast<int>(i) - static_cast<int>(ctr);
            const float xn = (static_cast<float>(xi) / (static_cast<float>(size) - 1.0f)) / fill;
            out[i] = expf(-10.0f * (xn * xn));
            continue;
        }
        const int xi = static_cast<int>(i) - min_pos;
        const float xn = static_cast<float>(xi) / wm1;
        if (xn > 0.999f || xn < 0.0001f) {
            out[i] = 0.0f;
            continue;
        }
        const double xd = static_cast<double>(xn);
        switch (type) {
            case 0:  // HANN
                out[i] = static_cast<float>(0.5 * (1.0 - std::cos(2.0 * kPi * xd)));
                break;
            case 2:  // SINE
                out[i] = static_cast<float>(std::sin(kPi * xd));
                break;
            case 3: {  // LANCZOS
                const float arg = 2.0f * xn - 1.0f;
                if (arg == 0.0f) {
                    out[i] = 1.0f;
                } else {
                    const double ad = static_cast<double>(arg);
                    out[i] = static_cast<float>(std::sin(kPi * ad) / (kPi * ad));
                }
                break;
            }
            case 4:  // RECTANGULAR
                out[i] = 1.0f;
                break;
            default: {  // FLAT_TOP
                const float a0 = 0.215578948f, a1 = 0.416631580f, a2 = 0.277263158f, a3 = 0.083578947f,
                            a4 = 0.006947368f;
                out[i] = a0 - a1 * static_cast<float>(std::cos(2.0 * kPi * xd)) +
                         a2 * static_cast<float>(std::cos(4.0 * kPi * xd)) -
                         a3 * static_cast<float>(std::cos(6.0 * kPi * xd)) +
                         a4 * static_cast<float>(std::cos(8.0 * kPi * xd));
                break;
            }
        }
    }
    return OPE_B200_OK;
}

// Phase -> interleaved (cos, sin) with float cosf/sinf, the hand-off of
// Processor::Impl::getDispersionCurve (src/core/processor.cpp:91-98).
int ope_b200_phase_to_cos_sin(const float* phase, size_t n, float* out) {
    if (!phase || !out) return OPE_B200_E_INVALID;
    for (size_t i = 0; i < n; ++i) {
        out[2 * i] = cosf(phase[i]);
        out[2 * i + 1] = sinf(phase[i]);
    }
    return OPE_B200_OK;
}

}  // extern "C"
