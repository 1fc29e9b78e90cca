// CPU emulation of the fused chain kernel. TEST INFRASTRUCTURE ONLY.
//
// Runs the kernel's own __host__ __device__ phase functions
// (octproengine_b200/csrc/chain_kernel.cuh) for every thread of a team,
// phase by phase, with the same shared-memory layout and with every shared
// memory index bounds-checked (OPE_SMEM_CHECK asserts in the host build). It
// lets the CPU test suite check the kernels' index arithmetic, the
// bit-exactness of the pre-FFT stages and the FFT itself without a GPU. It is
// never linked into the product.
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../octproengine_b200/csrc/chain_kernel.cuh"
#include "../../octproengine_b200/csrc/tables.h"

using namespace ope_b200;

extern "C" {
struct EmuArgs {
    int n, in_kind, interp;
    long long m;
    const void* in;
    const float* curve;
    const float* window;
    const float* cos_sin;
    const float* fpn;  // interleaved n/2 pairs or null
    int dc_window;
    int log_scaling;
    float gmin, gmax, addend, mult;
    int flip, ascans_per_bscan, bscans;
    int dc_split;
    int dc_ref_order;
};
}

namespace {

enum { OUT_IMAGE = 0, OUT_FFT_INPUT = 1, OUT_BINS = 2, OUT_RESAMPLED = 3 };

// The kernel's reference-order shortcut: integer samples whose two row
// totals (exact) keep every float partial sum exact take the exact-sum path.
template <int N, int DT>
bool ref_order_exact(const unsigned char* stage) {
    if (DT == IN_F32) return false;
    using sum_t = typename InTraits<DT>::sum_t;
    sum_t ta = 0, tb = 0;
    for (int t = 0; t < N / 16; ++t) {
        sum_t a, b;
        phase_dc_local<N, DT>(t, stage, &a, &b);
        ta += a;
        tb += b;
    }
    return dc_prefix_exact_in_float(ta) && dc_prefix_exact_in_float(tb);
}

template <int N, int DT, int INTERP>
int emu_run(const EmuArgs& e, int what, float* out) {
    using PL = Plan<N>;
    using LY = Layout<N, DT>;
    using sum_t = typename InTraits<DT>::sum_t;
    using raw_t = typename InTraits<DT>::raw_t;
    constexpr int T = PL::T;
    constexpr int NPASS = PL::NPASS;

    std::vector<float2> tw = build_twiddles(N);
    std::vector<int2> lin;
    std::vector<int2> cub;
    std::vector<int> lzb;
    std::vector<float> lzw;
    if (INTERP == INTERP_LINEAR) lin = build_linear_table(e.curve, N);
    if (INTERP == INTERP_CUBIC) cub = build_cubic_table(e.curve, N);
    if (INTERP == INTERP_LANCZOS) build_lanczos_table(e.curve, N, lzb, lzw);
    std::vector<float2> wph = build_window_phase(e.window, e.cos_sin, N);
    std::vector<float2> dcr;
    if (e.dc_split && e.dc_window == 0)
        dcr = build_dc_response(N, INTERP, lzw.empty() ? nullptr : lzw.data(), e.window, e.cos_sin);

    ChainArgs a{};
    a.in = e.in;
    a.m = e.m;
    a.tw = tw.data();
    a.lin = lin.data();
    a.cub = cub.data();
    a.lz_base = lzb.data();
    a.lz_w = lzw.data();
    a.wph = wph.data();
    a.fpn = reinterpret_cast<const float2*>(e.fpn);
    a.dc_window = e.dc_window;
    scaling_constants(e.log_scaling != 0, e.gmin, e.gmax, e.addend, e.mult, N, a);
    a.flip = e.flip;
    a.ascans_per_bscan = e.ascans_per_bscan;
    a.bscans = e.bscans;
    a.neg_zero = -0.0f;
    a.dc_resp = dcr.empty() ? nullptr : dcr.data();

    std::vector<unsigned char> work(LY::WORK_BYTES + 64, 0);
    std::vector<unsigned char> stage(LY::STAGE_BYTES, 0);
    float2* spec = reinterpret_cast<float2*>(work.data() + LY::OFF_SPEC);
    float4* exch = reinterpret_cast<float4*>(work.data() + LY::OFF_EXCH);
    sum_t* pfx = reinterpret_cast<sum_t*>(work.data() + LY::OFF_PFX);
    std::vector<std::array<cp, 16>> v(T);
    const size_t row_bytes = N * sizeof(raw_t);
    const unsigned char* in = static_cast<const unsigned char*>(e.in);

    // 8/16-bit samples without rolling-average DC removal: the kernel keeps the
    // spectrum as packed integer words (phase_store_packed) and interpolates
    // from them (phase_prestage_packed); the emulation runs the same phases
    constexpr bool PACKABLE = (DT == IN_U8 || DT == IN_U16);
    const bool packed = PACKABLE && e.dc_window == 0;
    float2 cbias = make_float2(8388608.0f, 8388608.0f);

    for (long long r = 0; r < e.m; r += 2) {
        const bool has_b = r + 1 < e.m;
        std::memcpy(stage.data(), in + r * row_bytes, row_bytes * (has_b ? 2 : 1));
        if (!has_b) std::memset(stage.data() + row_bytes, 0, row_bytes);
        float2 dc = make_float2(0.0f, 0.0f);
        cbias = make_float2(8388608.0f, 8388608.0f);
        if (packed) {
            std::vector<std::array<uint32_t, 16>> words(T);
            long long ta = 0, tb = 0;  // exact integer sums: any order
            for (int t = 0; t < T; ++t) {
                int sa = 0, sb = 0;
                phase_split_load_packed<N, DT>(t, stage.data(), words[t].data(), &sa, &sb);
                ta += sa;
                tb += sb;
            }
            if (a.dc_resp) {
                dc = make_float2(split_level((double)ta, N, true), split_level((double)tb, N, true));
                cbias = add2(cbias, dc);
            }
            for (int t = 0; t < T; ++t) phase_store_packed<N>(t, words[t].data(), reinterpret_cast<uint32_t*>(spec));
        } else if (e.dc_window == 0 && a.dc_resp) {
            // same reduction tree as team_sum2: xor butterfly per warp, lane 0, then warps in order
            using SS = typename SplitSum<DT>::type;
            std::vector<std::array<float2, 16>> vals(T);
            std::vector<SS> sa(T), sb(T);
            for (int t = 0; t < T; ++t) phase_split_load<N, DT>(t, stage.data(), vals[t].data(), &sa[t], &sb[t]);
            SS ta = 0, tb = 0;
            for (int w = 0; w < T / 32; ++w) {
                std::array<SS, 32> xa, xb;
                for (int l = 0; l < 32; ++l) {
                    xa[l] = sa[32 * w + l];
                    xb[l] = sb[32 * w + l];
                }
                for (int o = 16; o > 0; o >>= 1) {
                    std::array<SS, 32> ya = xa, yb = xb;
                    for (int l = 0; l < 32; ++l) {
                        ya[l] = xa[l] + xa[l ^ o];
                        yb[l] = xb[l] + xb[l ^ o];
                    }
                    xa = ya;
                    xb = yb;
                }
                ta += xa[0];
                tb += xb[0];
            }
            dc = make_float2(split_level((double)ta, N, DT != IN_F32), split_level((double)tb, N, DT != IN_F32));
            for (int t = 0; t < T; ++t) phase_split_store<N>(t, vals[t].data(), dc, spec);
        } else if (e.dc_window > 0 && e.dc_ref_order && !ref_order_exact<N, DT>(stage.data())) {
            float* pf = reinterpret_cast<float*>(pfx);
            if constexpr (DT == IN_U16) {
                // the kernel's segment form of the float prefix: exact integer
                // prefixes per thread (any order), then its three steps in turn
                std::vector<int> ta(T), tb(T);
                int pa = 0, pb = 0;
                for (int t = 0; t < T; ++t) {
                    int a0, b0;
                    phase_dc_local<N, DT>(t, stage.data(), &a0, &b0);
                    ta[t] = pa;
                    tb[t] = pb;
                    pa += a0;
                    pb += b0;
                }
                static_assert(RefparArea<N>::BYTES <= LY::SPEC_BYTES, "the step records fit the spectrum area");
                unsigned char* area = work.data() + LY::OFF_SPEC;
                for (int t = 0; t < T; ++t) phase_dc_refpar_seg<N>(t, stage.data(), ta[t & ~3], tb[t & ~3], area);
                for (int t = 0; t < T; ++t) phase_dc_refpar_walk<N>(t, stage.data(), area);
                for (int t = 0; t < T; ++t) phase_dc_refpar_fill<N>(t, stage.data(), area, pf);
            } else {
                for (int t = 0; t < T; ++t) phase_dc_ref_scan<N, DT>(t, stage.data(), pf);
            }
            for (int t = 0; t < T; ++t) phase_dc_apply<N, DT, true>(t, stage.data(), pf, e.dc_window, spec);
        } else if (e.dc_window > 0) {
            // exact sums; also the reference order when every float partial sum is exact
            std::vector<sum_t> ta(T), tb(T);
            for (int t = 0; t < T; ++t) phase_dc_local<N, DT>(t, stage.data(), &ta[t], &tb[t]);
            // same order as team_exclusive_scan2: Hillis-Steele inclusive scan per
            // warp (shfl_up by 1, 2, 4, 8, 16), warp totals added in warp order
            {
                std::vector<sum_t> ia(ta), ib(tb);
                for (int w = 0; w < T / 32; ++w)
                    for (int o = 1; o < 32; o <<= 1) {
                        std::vector<sum_t> na(ia.begin() + 32 * w, ia.begin() + 32 * w + 32);
                        std::vector<sum_t> nb(ib.begin() + 32 * w, ib.begin() + 32 * w + 32);
                        for (int l = o; l < 32; ++l) {
                            na[l] = ia[32 * w + l] + ia[32 * w + l - o];
                            nb[l] = ib[32 * w + l] + ib[32 * w + l - o];
                        }
                        for (int l = 0; l < 32; ++l) {
                            ia[32 * w + l] = na[l];
                            ib[32 * w + l] = nb[l];
                        }
                    }
                for (int t = 0; t < T; ++t) {
                    const int w = t / 32;
                    sum_t pa = 0, pb = 0;
                    for (int u = 0; u < w; ++u) {
                        pa += ia[32 * u + 31];
                        pb += ib[32 * u + 31];
                    }
                    const sum_t xa = ta[t], xb = tb[t];
                    ta[t] = pa + ia[t] - xa;
                    tb[t] = pb + ib[t] - xb;
                }
            }
            for (int t = 0; t < T; ++t) phase_dc_prefix<N, DT>(t, stage.data(), ta[t], tb[t], pfx);
            for (int t = 0; t < T; ++t) phase_dc_apply<N, DT>(t, stage.data(), pfx, e.dc_window, spec);
        } else {
            for (int t = 0; t < T; ++t) phase_unpack<N, DT>(t, stage.data(), spec);
        }
        std::vector<float> rs;
        if (what == OUT_RESAMPLED) {
            rs.assign(2 * N, 0.0f);
            a.resampled_out = rs.data();
        }
        for (int t = 0; t < T; ++t) {
            if (packed)
                phase_prestage_packed<N, INTERP>(t, reinterpret_cast<const uint32_t*>(spec), cbias, a, v[t].data());
            else
                phase_prestage<N, INTERP>(t, spec, a, v[t].data());
        }
        a.resampled_out = nullptr;
        if (what == OUT_RESAMPLED) {
            for (int j = 0; j < N; ++j) {
                out[r * N + j] = rs[2 * j];
                if (has_b) out[(r + 1) * N + j] = rs[2 * j + 1];
            }
            continue;
        }
        if (what == OUT_FFT_INPUT) {
            for (int t = 0; t < T; ++t)
                for (int s = 0; s < 16; ++s) {
                    const int j = t + s * T;
                    const cp x = v[t][s];
                    out[(r * N + j) * 2] = x.re.x;
                    out[(r * N + j) * 2 + 1] = x.im.x;
                    if (has_b) {
                        out[((r + 1) * N + j) * 2] = x.re.y;
                        out[((r + 1) * N + j) * 2 + 1] = x.im.y;
                    }
                }
            continue;
        }
        for (int t = 0; t < T; ++t) fft_twiddle_dft<N, 0>(t, v[t].data(), tw.data());
        for (int t = 0; t < T; ++t) fft_store<N, 0>(t, v[t].data(), exch);
        if constexpr (NPASS > 2) {
            for (int t = 0; t < T; ++t) {
                fft_load<N>(t, exch, v[t].data());
                fft_twiddle_dft<N, 1>(t, v[t].data(), tw.data());
            }
            for (int t = 0; t < T; ++t) fft_store<N, 1>(t, v[t].data(), exch);
        }
        if constexpr (NPASS > 3) {
            for (int t = 0; t < T; ++t) {
                fft_load<N>(t, exch, v[t].data());
                fft_twiddle_dft<N, 2>(t, v[t].data(), tw.data());
            }
            for (int t = 0; t < T; ++t) fft_store<N, 2>(t, v[t].data(), exch);
        }
        for (int t = 0; t < T; ++t) {
            fft_load<N>(t, exch, v[t].data());
            fft_twiddle_dft<N, NPASS - 1>(t, v[t].data(), tw.data());
        }
        using L = LastInfo<N>;
        if (what == OUT_BINS) {
            for (int t = 0; t < T; ++t)
                for (int i = 0; i < L::D; ++i)
                    for (int q = 0; q < L::R / 2; ++q) {
                        const int bin = L::bin(t, i, q);
                        cp x = add_dc(a, v[t][i + q * L::D], bin, dc);
                        if (a.fpn) {
                            x.re = sub2(x.re, dup2(a.fpn[bin].x));
                            x.im = sub2(x.im, dup2(a.fpn[bin].y));
                        }
                        out[(r * (N / 2) + bin) * 2] = x.re.x;
                        out[(r * (N / 2) + bin) * 2 + 1] = x.im.x;
                        if (has_b) {
                            out[((r + 1) * (N / 2) + bin) * 2] = x.re.y;
                            out[((r + 1) * (N / 2) + bin) * 2 + 1] = x.im.y;
                        }
                    }
            continue;
        }
        // image epilogue (host restatement of the device epilogue; log2 is exact here)
        std::vector<float> img(2 * (N / 2));
        for (int t = 0; t < T; ++t) {
            float2 mag2[L::NB];
            epi_mag2<N>(t, v[t].data(), a, dc, mag2);
            for (int i = 0; i < L::D; ++i)
                for (int q = 0; q < L::R / 2; ++q) {
                    const int bin = L::bin(t, i, q);
                    const float2 m2 = mag2[i * (L::R / 2) + q];
                    img[bin] = a.log_mode ? std::log2(m2.x) : std::sqrt(m2.x);
                    img[N / 2 + bin] = a.log_mode ? std::log2(m2.y) : std::sqrt(m2.y);
                }
        }
        for (int lane = 0; lane < (has_b ? 2 : 1); ++lane) {
            float* row = img.data() + lane * (N / 2);
            if (a.log_mode && a.auto_minmax) {
                const double c10 = 10.0 * std::log10(2.0);
                float mn = INFINITY, mx = -INFINITY;
                for (int b = 0; b < N / 2; ++b) {
                    row[b] = static_cast<float>(c10 * row[b] - 10.0 * std::log10(N / 2.0));
                    mn = std::fmin(mn, row[b]);
                    mx = std::fmax(mx, row[b]);
                }
                float rg = mx - mn;
                if (!(rg >= 1e-6f)) rg = 1.0f;
                for (int b = 0; b < N / 2; ++b) row[b] = a.mult * ((row[b] - mn) / rg + a.addend);
            } else {
                for (int b = 0; b < N / 2; ++b) row[b] = std::fma(row[b], a.k_a, a.k_b);
            }
            const long long orow = out_row(a, r + lane);
            std::memcpy(out + orow * (N / 2), row, sizeof(float) * (N / 2));
        }
    }
    return 0;
}

template <int N, int DT>
int by_interp(const EmuArgs& e, int what, float* out) {
    switch (e.interp) {
        case INTERP_NONE: return emu_run<N, DT, INTERP_NONE>(e, what, out);
        case INTERP_LINEAR: return emu_run<N, DT, INTERP_LINEAR>(e, what, out);
        case INTERP_CUBIC: return emu_run<N, DT, INTERP_CUBIC>(e, what, out);
        case INTERP_LANCZOS: return emu_run<N, DT, INTERP_LANCZOS>(e, what, out);
    }
    return -1;
}

template <int N>
int by_dt(const EmuArgs& e, int what, float* out) {
    switch (e.in_kind) {
        case IN_U8: return by_interp<N, IN_U8>(e, what, out);
        case IN_U16: return by_interp<N, IN_U16>(e, what, out);
        case IN_U32: return by_interp<N, IN_U32>(e, what, out);
        case IN_F32: return by_interp<N, IN_F32>(e, what, out);
    }
    return -1;
}

}  // namespace

extern "C" int emu_chain(const EmuArgs* e, int what, float* out) {
    switch (e->n) {
        case 512: return by_dt<512>(*e, what, out);
        case 1024: return by_dt<1024>(*e, what, out);
        case 2048: return by_dt<2048>(*e, what, out);
        case 4096: return by_dt<4096>(*e, what, out);
        case 8192: return by_dt<8192>(*e, what, out);
    }
    return -1;
}
