// Host-side table builders (see tables.h). Compiled without FP contraction so
// the float expressions round exactly as the reference's do.
#include "tables.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <utility>

namespace ope_b200 {

namespace {

int trunc_index(float v) {
    // static_cast<int>(float) truncates toward zero; non-finite or huge values
    // (undefined in C++) are pinned so every table index stays in bounds.
    if (!(v == v)) return 0;
    if (v > 1.0e8f) return 100000000;
    if (v < -1.0e8f) return -100000000;
    return static_cast<int>(v);
}

int float_bits(float f) {
    int b;
    std::memcpy(&b, &f, 4);
    return b;
}

}  // namespace

float lanczos8(float x) {
    if (std::fabs(x) < 1e-5f) return 1.0f;
    if (std::fabs(x) >= 8.0f) return 0.0f;
    const float pi = static_cast<float>(3.14159265358979323846);
    const float px = pi * x;
    const float pa = px / 8.0f;
    return (sinf(px) / px) * (sinf(pa) / pa);
}

std::vector<float2> build_twiddles(int n, int sched) {
    // Per Stockham pass p >= 1 (radix R, span NS): (R-1) x NS entries,
    // entry (r-1)*NS + k = W_N^(r k N/(NS R)), matching Sched::tw_off.
    // Every pass has radix 16 except one of radix lastr, run last (sched 0)
    // or as pass sched - 1 (sched >= 1).
    std::vector<float2> tw(n, make_float2(1.0f, 0.0f));
    int log2n = 0;
    while ((1 << log2n) < n) ++log2n;
    const int npass = (log2n + 3) / 4;
    const int lastr = 1 << (log2n - 4 * (npass - 1));
    int off = 0, ns = 1;
    for (int p = 0; p < npass; ++p) {
        const int r_p = (p == short_pass_of(npass, sched)) ? lastr : 16;
        if (p > 0) {
            const int stride = n / (ns * r_p);
            for (int r = 1; r < r_p; ++r)
                for (int k = 0; k < ns; ++k) {
                    const long long j = static_cast<long long>(r) * k * stride;
                    const double ang = 2.0 * 3.14159265358979323846 * static_cast<double>(j) / n;
                    tw[off + (r - 1) * ns + k] =
                        make_float2(static_cast<float>(std::cos(ang)), static_cast<float>(std::sin(ang)));
                }
            off += (r_p - 1) * ns;
        }
        ns *= r_p;
    }
    return tw;
}

std::vector<int2> build_linear_table(const float* curve, int n) {
    std::vector<int2> tab(n);
    for (int j = 0; j < n; ++j) {
        const float nx = curve[j];
        int n1 = trunc_index(nx);
        if (n1 > n - 1) n1 = n - 1;
        if (n1 < -SPEC_PAD) n1 = -SPEC_PAD;  // the reference would read out of bounds here
        const float fr = nx - static_cast<float>(n1);
        tab[j] = make_int2(n1 + SPEC_PAD, float_bits(fr));
    }
    return tab;
}

std::vector<int2> build_cubic_table(const float* curve, int n) {
    std::vector<int2> tab(n);
    auto cl = [n](int v) {
        if (v > n - 1) v = n - 1;
        if (v < -SPEC_PAD) v = -SPEC_PAD;
        return v;
    };
    for (int j = 0; j < n; ++j) {
        const float nx = curve[j];
        const int i1 = trunc_index(nx);
        // taps n2 = min(i1+1, n-1) and n3 = min(i1+2, n-1) are read as n1+1 and
        // n1+2: past n-1 (or below 0) the replicated-edge padding holds the
        // clamped sample, so only n0 = |i1-1| needs its own index
        const int n0 = cl(std::abs(i1 - 1)) + SPEC_PAD;
        const int n1r = cl(i1);
        const int n1 = n1r + SPEC_PAD;
        const float pos = nx - static_cast<float>(n1r);
        tab[j] = make_int2(n0 | (n1 << 16), float_bits(pos));
    }
    return tab;
}

void build_lanczos_table(const float* curve, int n, std::vector<int>& base, std::vector<float>& w) {
    base.assign(n, 0);
    w.assign(16 * static_cast<size_t>(n), 0.0f);
    for (int j = 0; j < n; ++j) {
        const float nx = curve[j];
        const int n0 = trunc_index(nx);
        for (int k = 0; k < 16; ++k) {
            int idx = n0 - 7 + k;
            if (idx < 0) idx = 0;
            if (idx >= n) idx = n - 1;
            w[static_cast<size_t>(k) * n + j] = lanczos8(nx - static_cast<float>(idx));
        }
        // Taps n0-7 .. n0+8 read the replicated edge padding when they leave
        // [0, n); pinning n0 to [-9, n+7] keeps them inside it and reads the
        // same clamped samples.
        int b = n0;
        if (b < -9) b = -9;
        if (b > n + 7) b = n + 7;
        base[j] = b - 7 + SPEC_PAD;
    }
}

namespace {

// In-place iterative radix-2 inverse DFT (exp(+i)), unnormalised, float64.
void idft_inplace(std::vector<double>& re, std::vector<double>& im) {
    const size_t n = re.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            std::swap(re[i], re[j]);
            std::swap(im[i], im[j]);
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len / 2;
        for (size_t k = 0; k < half; ++k) {
            const double ang = 2.0 * 3.14159265358979323846 * static_cast<double>(k) / static_cast<double>(len);
            const double wr = std::cos(ang), wi = std::sin(ang);
            for (size_t b = 0; b < n; b += len) {
                const size_t i0 = b + k, i1 = b + k + half;
                const double tr = re[i1] * wr - im[i1] * wi;
                const double ti = re[i1] * wi + im[i1] * wr;
                re[i1] = re[i0] - tr;
                im[i1] = im[i0] - ti;
                re[i0] += tr;
                im[i0] += ti;
            }
        }
    }
}

}  // namespace

std::vector<float2> build_dc_response(int n, int interp, const float* lanczos_w, const float* window,
                                      const float* cos_sin) {
    std::vector<double> re(n), im(n);
    for (int j = 0; j < n; ++j) {
        double g = 1.0;
        if (interp == INTERP_LANCZOS && lanczos_w) {
            g = 0.0;
            for (int k = 0; k < 16; ++k) g += static_cast<double>(lanczos_w[static_cast<size_t>(k) * n + j]);
        }
        const double w = window ? static_cast<double>(window[j]) : 1.0;
        const double c = cos_sin ? static_cast<double>(cos_sin[2 * j]) : 1.0;
        const double s = cos_sin ? static_cast<double>(cos_sin[2 * j + 1]) : 0.0;
        re[j] = g * w * c;
        im[j] = g * w * s;
    }
    idft_inplace(re, im);
    std::vector<float2> d(n / 2);
    for (int k = 0; k < n / 2; ++k) d[k] = make_float2(static_cast<float>(re[k]), static_cast<float>(im[k]));
    return d;
}

std::vector<float2> build_window_phase(const float* window, const float* cos_sin, int n) {
    std::vector<float2> t(n);
    for (int j = 0; j < n; ++j) {
        const double w = window ? static_cast<double>(window[j]) : 1.0;
        const float wc = static_cast<float>(w * (cos_sin ? static_cast<double>(cos_sin[2 * j]) : 1.0));
        const float ws = static_cast<float>(w * (cos_sin ? static_cast<double>(cos_sin[2 * j + 1]) : 0.0));
        t[j] = make_float2(wc, ws);
    }
    return t;
}

void scaling_constants(bool log_scaling, float gmin_f, float gmax_f, float addend_f, float mult_f, int n,
                       ChainArgs& a) {
    const double half = n / 2;
    const double mult = mult_f, addend = addend_f, gmin = gmin_f;
    // range in float as the reference computes it (cpu_kernels.tpp:332-335,356-361)
    float rf = gmax_f - gmin_f;
    if (rf < 1e-6f) rf = 1.0f;
    const double range = rf;
    a.mult = mult_f;
    a.addend = addend_f;
    if (log_scaling) {
        // out = mult*((10 log10(|X|^2/(N/2)) - min)/range + addend)
        const double c10 = 10.0 * std::log10(2.0);
        a.log_mode = 1;
        a.auto_minmax = (gmin_f == gmax_f) ? 1 : 0;
        a.k_a = static_cast<float>(mult * c10 / range);
        a.k_b = static_cast<float>(mult * ((-10.0 * std::log10(half) - gmin) / range + addend));
    } else {
        // out = mult*((|X|/(N/2) - min)/range + addend)
        a.log_mode = 0;
        a.auto_minmax = 0;
        a.k_a = static_cast<float>(mult / (half * range));
        a.k_b = static_cast<float>(mult * (addend - gmin / range));
    }
}

}  // namespace ope_b200
