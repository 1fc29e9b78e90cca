// Differentiable chain for dispersion / k-mapping autofocus (sm_100a).
//
// Parameters (device float[8]): the dispersion polynomial d0..d3 and the
// resampling polynomial c0..c3 in the reference convention
// (src/core/processorconfiguration.cpp:438-482): with t = j/(N-1),
//   r(j)   = clamp(sum_m c_m t^m, 7, N-9)   raw position of output sample j
//   phi(j) = sum_m d_m t^m                  dispersion phase
// The forward chain per A-scan is the reference's (cpu_backend.cpp:184-264)
// with the tables built on the device from the parameters:
//   x - c (c = the A-scan's integer mean, subtracted exactly and not added
//   back: autofocus scores the image without its DC term)
//   y_j = interp(x - c; r_j)                    linear, cubic or Lanczos-8
//   z_j = y_j * w_j * exp(i phi_j)
//   X_k = sum_j z_j exp(+2 pi i j k / N), k < N/2      (unnormalised inverse DFT)
//   I_k = |X_k|^2
// The adjoint (af_backward_kernel) recomputes this forward instead of storing
// complex intermediates, then runs, per pair of A-scans:
//   dL/dX_k = 2 G_k X_k  (G_k = dL/dI_k; for the entropy objective
//             G_k = -(ln(I_k/S) + H)/S, for a dB output G_k = G_out 10/(ln10 I_k))
//   a = F u, u_k = conj(dL/dX_k)          the adjoint DFT, as a second inverse DFT
//   h_j = a_j * w_j * exp(i phi_j)
//   dL/dy_j   = Re h_j                    adjoint of the window/phase product
//   dL/dphi_j = -y_j Im h_j               adjoint of the phase
//   dL/dd_m = sum_j t_j^m dL/dphi_j
//   dL/dc_m = sum_j t_j^m dL/dy_j dy_j/dr_j  (0 where r_j is clamped)
// dy/dr is the derivative of the interpolation kernel (the transpose of the
// resampling with respect to the sample positions).
#pragma once

#include "chain_device.cuh"

namespace ope_b200 {

constexpr int AF_NPARAM = 8;  // d0..d3, c0..c3
constexpr int AF_OUT_NONE = 0, AF_OUT_INTENSITY = 1, AF_OUT_DB = 2;

struct AfArgs {
    ChainArgs c;             // input, A-scan count, twiddles, device-built tables
    const float* lz_dw;      // LANCZOS: 16 x N derivative weights dL(x)/dx, tap-major
    const float* rmask;      // 1 where r_j lies inside [7, N-9], else 0
    float* out;              // forward output (M x N/2) or nullptr
    int out_mode;            // AF_OUT_*
    const float* grad_out;   // backward: dL/d(out), M x N/2; nullptr = entropy objective
    const double* hs;        // entropy objective: hs[0] = H, hs[1] = S
    double* partial;         // per-CTA partial sums (forward: 2, backward: 8 per CTA)
    int disp_only;           // backward: dispersion gradients only (k-map entries left 0)
};

// ------------------------------------------------------------ tables ----

// lanczosKernel<float>(x, 8) of the reference (cpu_kernels.tpp:148-162) with
// the device's sinf, and its derivative in double.
__device__ __forceinline__ float af_lanczos8(float x) {
    if (fabsf(x) < 1e-5f) return 1.0f;
    if (fabsf(x) >= 8.0f) return 0.0f;
    const float pi = 3.14159265358979323846f;
    const float px = __fmul_rn(pi, x);
    const float pa = __fdiv_rn(px, 8.0f);
    return __fmul_rn(__fdiv_rn(sinf(px), px), __fdiv_rn(sinf(pa), pa));
}

__device__ __forceinline__ float af_lanczos8_deriv(float xf) {
    const double x = xf;
    if (fabs(x) < 1e-5 || fabs(x) >= 8.0) return 0.0f;
    const double a = 3.14159265358979323846 * x, b = a / 8.0;
    double sa, ca, sb, cb;
    sincos(a, &sa, &ca);
    sincos(b, &sb, &cb);
    const double f1 = sa / a, f2 = sb / b;
    // d/dx sinc(x) = (cos(pi x) - sinc(x)) / x; d/dx sinc(x/8) = (cos(pi x/8) - sinc(x/8)) / x
    return static_cast<float>((ca - f1) / x * f2 + f1 * (cb - f2) / x);
}

// The device tables of one evaluation, in one launch: one thread per output
// sample j for the resampling tables, window x phase factors and the clamp
// mask, then (Lanczos-8) one thread per (tap, sample) for the tap weights,
// all from the device parameter vector. The polynomials are
// evaluated as generateResamplingCurve / generateDispersionCurve do
// (processorconfiguration.cpp:438-482): float Horner in j with the
// coefficients divided by (N-1)^m, every operation rounded separately.
__global__ void af_prepare_kernel(int n, int interp, int tb, const float* __restrict__ params,
                                  const float* __restrict__ window, int2* lin, int2* cub, int* lzb, float* lzw,
                                  float* lzdw, float* rmask, float2* wph);

// ------------------------------------------------------------ forward ----

template <int N>
struct AfForwardSink {
    const AfArgs* args;
    double s = 0.0, e = 0.0;  // sum I, sum I ln I over this CTA's bins
    __device__ __forceinline__ void operator()(int t, const cp* v, long long row_a, bool has_b, float2) {
        using L = LastInfo<N>;
        const float ln2 = 0.69314718055994530942f;
        const float c10 = 3.01029995663981195214f;  // 10 log10(2)
        const float db_off = c10 * (float)(Plan<N>::LOG2N - 1);
#pragma unroll
        for (int i = 0; i < L::D; ++i)
#pragma unroll
            for (int q = 0; q < L::R / 2; ++q) {
                const int bin = L::bin(t, i, q);
                const cp x = v[i + q * L::D];
                const float2 I = fma2(x.re, x.re, mul2(x.im, x.im));
                const float2 lg = make_float2(__log2f(I.x), __log2f(I.y));
                if (args->out) {
                    float2 o = I;
                    if (args->out_mode == AF_OUT_DB) o = make_float2(c10 * lg.x - db_off, c10 * lg.y - db_off);
                    args->out[row_a * (N / 2) + bin] = o.x;
                    if (has_b) args->out[(row_a + 1) * (N / 2) + bin] = o.y;
                }
                s += (double)I.x;
                if (I.x > 0.0f) e += (double)(I.x * (lg.x * ln2));
                if (has_b) {
                    s += (double)I.y;
                    if (I.y > 0.0f) e += (double)(I.y * (lg.y * ln2));
                }
            }
    }
};

template <int N, int DT, int INTERP>
__global__ void __launch_bounds__(N / 16, 8192 / N) af_forward_kernel(const AfArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    using LY = Layout<N, DT>;
    AfForwardSink<N> sink;
    sink.args = &a;
    const long long npairs = (a.c.m + 1) / 2;
    const CtaTeam tm;
    run_pairs<N, DT, INTERP, 0>(tm, a.c, 0, a.c.m, blockIdx.x, npairs, gridDim.x, smem, sink);
    double s = sink.s, e = sink.e;
    team_sum2<N / 16, double>(tm, s, e, reinterpret_cast<double*>(smem + LY::OFF_SCAN));
    if (threadIdx.x == 0) {
        a.partial[2 * blockIdx.x] = s;
        a.partial[2 * blockIdx.x + 1] = e;
    }
}

// ----------------------------------------------------------- backward ----

template <int N, int DT>
struct AfLayout {
    using raw_t = typename InTraits<DT>::raw_t;
    static constexpr int ROW_BYTES = N * (int)sizeof(raw_t);
    // the spectrum overlays the raw rows: the unpack holds a pair's samples in
    // registers across the team sum before it writes the spectrum
    static constexpr int OFF_STAGE = 0;
    static constexpr int OFF_SPEC = 0;
    static constexpr int SPEC_OR_STAGE = (N + 2 * SPEC_PAD) * 8 > 2 * ROW_BYTES ? (N + 2 * SPEC_PAD) * 8 : 2 * ROW_BYTES;
    static constexpr int OFF_EXCH = ((SPEC_OR_STAGE + 127) / 128) * 128;
    static constexpr int OFF_SCAN = OFF_EXCH + Plan<N>::EXCH_ELEMS * 16;
    static constexpr int TOTAL = OFF_SCAN + 1024;
    static_assert(OFF_SPEC % 128 == 0 && OFF_EXCH % 128 == 0 && OFF_SCAN % 16 == 0,
                  "shared-memory regions must stay aligned for their widest accesses");
};

// Interpolated value alone (the dispersion-only adjoint), same arithmetic as
// af_interp_deriv's value.
template <int N, int INTERP>
__device__ __forceinline__ float2 af_interp_value(const float2* spec, const AfArgs& a, int j) {
    if (INTERP == INTERP_LINEAR) {
        const int2 e = a.c.lin[j];
        const float2 y1 = spec[e.x], y2 = spec[e.x + 1];
        return fma2(sub2(y2, y1), dup2(__int_as_float(e.y)), y1);
    } else if (INTERP == INTERP_CUBIC) {
        const int2 e = a.c.cub[j];
        const int i0 = e.x & 0xFFFF, i1 = (unsigned)e.x >> 16;
        const float pos = __int_as_float(e.y);
        const float2 y0 = spec[i0], y1 = spec[i1], y2 = spec[i1 + 1], y3 = spec[i1 + 2];
        const float2 ca = add2(sub2(mul2(dup2(3.0f), sub2(y1, y2)), y0), y3);
        const float2 cb = sub2(add2(sub2(mul2(dup2(2.0f), y0), mul2(dup2(5.0f), y1)), mul2(dup2(4.0f), y2)), y3);
        const float2 cc = sub2(y2, y0);
        const float2 P = dup2(pos);
        return fma2(mul2(dup2(0.5f * pos), fma2(fma2(ca, P, cb), P, cc)), dup2(1.0f), y1);
    } else if (INTERP == INTERP_LANCZOS) {
        const int b = a.c.lz_base[j];
        float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < 16; ++k) acc = fma2(spec[b + k], dup2(__ldg(a.c.lz_w + k * N + j)), acc);
        return acc;
    }
    return spec[SPEC_PAD + j];
}

// Interpolated value and its derivative with respect to the position, for
// both A-scans of a pair, at output sample j.
template <int N, int INTERP>
__device__ __forceinline__ void af_interp_deriv(const float2* spec, const AfArgs& a, int j, float2& y, float2& dy) {
    if (INTERP == INTERP_LINEAR) {
        const int2 e = a.c.lin[j];
        const float2 y1 = spec[e.x], y2 = spec[e.x + 1];
        const float fr = __int_as_float(e.y);
        dy = sub2(y2, y1);
        y = fma2(dy, dup2(fr), y1);
    } else if (INTERP == INTERP_CUBIC) {
        // y = y1 + pos/2 (cc + cb pos + ca pos^2); dy/dpos = cc/2 + cb pos + 3/2 ca pos^2
        const int2 e = a.c.cub[j];
        const int i0 = e.x & 0xFFFF, i1 = (unsigned)e.x >> 16;
        const float pos = __int_as_float(e.y);
        const float2 y0 = spec[i0], y1 = spec[i1], y2 = spec[i1 + 1], y3 = spec[i1 + 2];
        const float2 ca = add2(sub2(mul2(dup2(3.0f), sub2(y1, y2)), y0), y3);
        const float2 cb = sub2(add2(sub2(mul2(dup2(2.0f), y0), mul2(dup2(5.0f), y1)), mul2(dup2(4.0f), y2)), y3);
        const float2 cc = sub2(y2, y0);
        const float2 P = dup2(pos);
        y = fma2(mul2(dup2(0.5f * pos), fma2(fma2(ca, P, cb), P, cc)), dup2(1.0f), y1);
        dy = fma2(fma2(mul2(dup2(1.5f), ca), P, cb), P, mul2(dup2(0.5f), cc));
    } else if (INTERP == INTERP_LANCZOS) {
        const int b = a.c.lz_base[j];
        float2 acc = make_float2(0.0f, 0.0f), dacc = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const float2 s = spec[b + k];
            acc = fma2(s, dup2(__ldg(a.c.lz_w + k * N + j)), acc);
            dacc = fma2(s, dup2(__ldg(a.lz_dw + k * N + j)), dacc);
        }
        y = acc;
        dy = dacc;
    } else {
        y = spec[SPEC_PAD + j];
        dy = make_float2(0.0f, 0.0f);
    }
}

// Sums 8 values over the CTA in a fixed order (warp butterfly, then warps in
// order) and lets thread 0 write them to dst.
template <int T>
__device__ __forceinline__ void af_cta_sum8(const float* v, double* scratch, double* dst) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double d[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        d[m] = (double)v[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d[m] += __shfl_xor_sync(0xffffffffu, d[m], o);
    }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int m = 0; m < 8; ++m) scratch[warp * 8 + m] = d[m];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int m = 0; m < 8; ++m) {
            double s = 0.0;
            for (int w = 0; w < T / 32; ++w) s += scratch[w * 8 + m];
            dst[m] = s;
        }
    }
}

// CTAs per SM the adjoint's registers are capped for: 4 at N = 2048 (128
// registers; its shared memory also allows 4, so the 512 pairs of a
// 1024-A-scan B-scan take one round), 8 at N = 1024, 1 at N = 4096 (whose
// shared memory allows only one).
template <int N>
struct AfBwdOcc {
    static constexpr int MIN_BLOCKS = N <= 1024 ? 8 : N == 2048 ? 4 : 1;
};

template <int N, int DT, int INTERP>
__global__ void __launch_bounds__(N / 16, AfBwdOcc<N>::MIN_BLOCKS) af_backward_kernel(const AfArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    using PL = Plan<N>;
    using LY = AfLayout<N, DT>;
    using L = LastInfo<N>;
    using SS = typename SplitSum<DT>::type;
    constexpr int T = PL::T;
    constexpr int NPASS = PL::NPASS;
    unsigned char* stage = smem + LY::OFF_STAGE;
    float2* spec = reinterpret_cast<float2*>(smem + LY::OFF_SPEC);
    float4* exch = reinterpret_cast<float4*>(smem + LY::OFF_EXCH);
    double* scan = reinterpret_cast<double*>(smem + LY::OFF_SCAN);
    const int t = threadIdx.x;
    const ChainArgs& c = a.c;
    const long long m = c.m;
    const long long npairs = (m + 1) / 2;
    const float inv_nm1 = 1.0f / (float)(N - 1);

    float H = 0.0f, lnS = 0.0f, invS = 0.0f;
    if (!a.grad_out) {
        H = (float)a.hs[0];
        lnS = (float)log(a.hs[1]);
        invS = (float)(1.0 / a.hs[1]);
    }
    const float ln2 = 0.69314718055994530942f;
    const float db_k = 4.34294481903251827651f;  // 10 / ln 10

    float acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = 0.0f;

    for (long long pair = blockIdx.x; pair < npairs; pair += gridDim.x) {
        const long long row_a = 2 * pair;
        const bool has_b = row_a + 1 < m;
        // ---- raw rows -> shared (row b repeats row a when absent) ----
        {
            const uint4* src_a = reinterpret_cast<const uint4*>(static_cast<const unsigned char*>(c.in) +
                                                                 row_a * (long long)LY::ROW_BYTES);
            const uint4* src_b = has_b ? src_a + LY::ROW_BYTES / 16 : src_a;
            uint4* dst = reinterpret_cast<uint4*>(stage);
            for (int k = t; k < LY::ROW_BYTES / 16; k += T) {
                dst[k] = __ldg(src_a + k);
                dst[LY::ROW_BYTES / 16 + k] = __ldg(src_b + k);
            }
        }
        __syncthreads();
        if constexpr (DT == IN_U8 || DT == IN_U16) {
            if (c.bitshift) {  // as the forward applies it (run_pairs)
                phase_bitshift<N, DT>(t, stage);
                __syncthreads();
            }
        }
        // ---- x - c (exact integer mean) ----
        {
            float2 vals[16];
            SS sa, sb;
            phase_split_load<N, DT>(t, stage, vals, &sa, &sb);
            team_sum2<T, SS>(CtaTeam{}, sa, sb, reinterpret_cast<SS*>(scan));
            const float2 lvl = make_float2(split_level((double)sa, N, DT != IN_F32),
                                           split_level((double)sb, N, DT != IN_F32));
            phase_split_store<N>(t, vals, lvl, spec);
        }
        __syncthreads();
        // ---- recompute the forward up to X ----
        cp v[16];
        if (a.disp_only) {
            // the dispersion adjoint needs y, not dy/dr (recomputed below from the spectrum)
#pragma unroll
            for (int s2 = 0; s2 < 16; ++s2) {
                const int j = t + s2 * T;
                const float2 y = af_interp_value<N, INTERP>(spec, a, j);
                const float2 q = __ldg(c.wph + j);
                v[s2] = cpmake(mul2(y, dup2(q.x)), mul2(y, dup2(q.y)));
            }
        } else {
            phase_prestage<N, INTERP>(t, spec, c, v);
        }
        fft_twiddle_dft<N, 0>(t, v, c.tw);
        fft_store<N, 0>(t, v, exch);
        __syncthreads();
        if constexpr (NPASS > 2) {
            fft_load<N>(t, exch, v);
            fft_twiddle_dft<N, 1>(t, v, c.tw);
            __syncthreads();
            fft_store<N, 1>(t, v, exch);
            __syncthreads();
        }
        if constexpr (NPASS > 3) {
            fft_load<N>(t, exch, v);
            fft_twiddle_dft<N, 2>(t, v, c.tw);
            __syncthreads();
            fft_store<N, 2>(t, v, exch);
            __syncthreads();
        }
        fft_load<N>(t, exch, v);
        fft_twiddle_dft<N, NPASS - 1>(t, v, c.tw);
        // ---- u_k = conj(2 G_k X_k) for k < N/2, 0 above ----
        __syncthreads();  // every thread has read exch
#pragma unroll
        for (int i = 0; i < L::D; ++i)
#pragma unroll
            for (int q = 0; q < L::R / 2; ++q) {
                const int bin = L::bin(t, i, q);
                const cp x = v[i + q * L::D];
                const float2 I = fma2(x.re, x.re, mul2(x.im, x.im));
                float2 G;
                if (a.grad_out) {
                    G.x = a.grad_out[row_a * (N / 2) + bin];
                    G.y = has_b ? a.grad_out[(row_a + 1) * (N / 2) + bin] : 0.0f;
                    if (a.out_mode == AF_OUT_DB) G = make_float2(G.x * db_k / I.x, G.y * db_k / I.y);
                } else {
                    // entropy H = -sum p ln p, p = I/S: dH/dI = -(ln p + H)/S
                    G.x = -(__log2f(I.x) * ln2 - lnS + H) * invS;
                    G.y = has_b ? -(__log2f(I.y) * ln2 - lnS + H) * invS : 0.0f;
                }
                if (!(I.x > 0.0f)) G.x = 0.0f;
                if (!(I.y > 0.0f)) G.y = 0.0f;
                const float2 g2 = mul2(G, dup2(2.0f));
                const float2 ure = mul2(g2, x.re), uim = neg2(mul2(g2, x.im));
                exch[xslot(bin)] = make_float4(ure.x, ure.y, uim.x, uim.y);
                exch[xslot(bin + N / 2)] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        __syncthreads();
        // ---- adjoint DFT: a = F u (all N outputs) ----
        fft_load<N>(t, exch, v);
        fft_twiddle_dft<N, 0, (NPASS == 1)>(t, v, c.tw);
        __syncthreads();
        fft_store<N, 0>(t, v, exch);
        __syncthreads();
        if constexpr (NPASS > 2) {
            fft_load<N>(t, exch, v);
            fft_twiddle_dft<N, 1>(t, v, c.tw);
            __syncthreads();
            fft_store<N, 1>(t, v, exch);
            __syncthreads();
        }
        if constexpr (NPASS > 3) {
            fft_load<N>(t, exch, v);
            fft_twiddle_dft<N, 2>(t, v, c.tw);
            __syncthreads();
            fft_store<N, 2>(t, v, exch);
            __syncthreads();
        }
        fft_load<N>(t, exch, v);
        fft_twiddle_dft<N, NPASS - 1, true>(t, v, c.tw);
        // ---- per-sample adjoints, reduced onto the 8 parameters ----
        using PI = PassInfo<N, NPASS - 1>;
#pragma unroll
        for (int i = 0; i < PI::D; ++i)
#pragma unroll
            for (int q = 0; q < PI::R; ++q) {
                const int j = t + i * T + q * (N / PI::R);
                const cp A = v[i + q * PI::D];
                const float2 w = __ldg(c.wph + j);
                const float2 wc = dup2(w.x), ws = dup2(w.y);
                const float2 hre = fma2(A.re, wc, neg2(mul2(A.im, ws)));
                const float2 him = fma2(A.re, ws, mul2(A.im, wc));
                float2 y, dy;
                float gr = 0.0f;
                if (a.disp_only) {
                    y = af_interp_value<N, INTERP>(spec, a, j);
                } else {
                    af_interp_deriv<N, INTERP>(spec, a, j, y, dy);
                    const float2 gy2 = mul2(hre, dy);
                    gr = (gy2.x + gy2.y) * __ldg(a.rmask + j);
                }
                const float2 gphi2 = neg2(mul2(y, him));
                const float gphi = gphi2.x + gphi2.y;
                const float tj = (float)j * inv_nm1;
                float p = 1.0f;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    acc[k] = fmaf(p, gphi, acc[k]);
                    acc[4 + k] = fmaf(p, gr, acc[4 + k]);
                    p *= tj;
                }
            }
        __syncthreads();  // the next pair overwrites stage, spec and exch
    }
    af_cta_sum8<T>(acc, scan, a.partial + 8 * (long long)blockIdx.x);
}

}  // namespace ope_b200
