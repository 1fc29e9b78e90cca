// Low-level per-operation API (ProcessingBackend, backend_interface.h:50-164;
// Processor, include/processor.h:165-282): each stage of the chain on its own,
// on host arrays, for unit-level checks. The reference CPU backend implements
// convertInput, kLinearization, windowing, dispersionCompensation, ifft,
// getMinimumVarianceMean and fixedPatternNoiseRemoval (cpu_backend.cpp:514-
// 733) and returns zero vectors for the rest; its CUDA backend returns empty
// results for all (cuda_backend.cu:1133-1296). Here every operation runs as a
// GPU kernel; the ones the CPU backend implements follow its kernels'
// arithmetic (cpu_kernels.tpp), the others follow the chain's semantics.
// Calls are synchronous: copy in, one kernel, copy out.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/ope_b200.h"
#include "autofocus.cuh"
#include "postproc.h"
#include "tables.h"

namespace ope_b200 {
namespace {

constexpr int kThreads = 256;

unsigned blocks_for(long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    if (b > 148 * 64) b = 148 * 64;
    return b < 1 ? 1u : (unsigned)b;
}

__global__ void op_convert_kernel(const void* in, int bit_depth, long long n, float* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (bit_depth <= 8) out[i] = (float)static_cast<const uint8_t*>(in)[i];
        else if (bit_depth <= 16) out[i] = (float)static_cast<const uint16_t*>(in)[i];
        else out[i] = __uint2float_rn(static_cast<const uint32_t*>(in)[i]);
    }
}

// kLinearization{Linear,Cubic,Lanczos} (cpu_kernels.tpp:84-196) on one line
// of n_in samples; indices clamped to [0, n_in-1] (the reference clamps only
// from above).
__global__ void op_klin_kernel(const float* in, int n_in, const float* curve, int method, int width, float* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= width) return;
    const float nx = curve[j];
    auto at = [&](int q) { return in[q < 0 ? 0 : (q > n_in - 1 ? n_in - 1 : q)]; };
    const int t = (nx == nx) ? (int)nx : 0;
    if (method == 0) {
        const int n1 = t < n_in - 1 ? t : n_in - 1;
        const float y1 = at(n1), y2 = at(t + 1 < n_in - 1 ? t + 1 : n_in - 1);
        out[j] = __fadd_rn(y1, __fmul_rn(__fsub_rn(y2, y1), __fsub_rn(nx, (float)n1)));
    } else if (method == 1) {
        const int n1 = t < n_in - 1 ? t : n_in - 1;
        const int n0 = abs(t - 1);
        const float y0 = at(n0 < n_in - 1 ? n0 : n_in - 1), y1 = at(n1);
        const float y2 = at(t + 1 < n_in - 1 ? t + 1 : n_in - 1), y3 = at(t + 2 < n_in - 1 ? t + 2 : n_in - 1);
        const float a = __fadd_rn(__fadd_rn(-y0, __fmul_rn(3.0f, __fsub_rn(y1, y2))), y3);
        const float b = __fsub_rn(__fadd_rn(__fsub_rn(__fmul_rn(2.0f, y0), __fmul_rn(5.0f, y1)), __fmul_rn(4.0f, y2)), y3);
        const float c = __fadd_rn(-y0, y2);
        const float pos = __fsub_rn(nx, (float)n1);
        const float pos2 = __fmul_rn(pos, pos);
        const float in_ = __fadd_rn(__fadd_rn(__fmul_rn(a, pos2), __fmul_rn(b, pos)), c);
        out[j] = __fadd_rn(__fmul_rn(__fmul_rn(0.5f, pos), in_), y1);
    } else {
        float sum = 0.0f;
        for (int i = -7; i <= 8; ++i) {
            int idx = t + i;
            idx = idx < 0 ? 0 : (idx >= n_in ? n_in - 1 : idx);
            sum = __fadd_rn(sum, __fmul_rn(in[idx], af_lanczos8(__fsub_rn(nx, (float)idx))));
        }
        out[j] = sum;
    }
}

// Per element: window (mode 1), real part of the dispersion product (mode 2),
// dispersion then window (mode 3: real part of (x * phase) * w).
__global__ void op_elementwise_kernel(const float* in, const float* win, const float* cs, int mode, long long n,
                                      float* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float v = in[i];
        if (mode & 2) v = __fmul_rn(v, cs[2 * i]);
        if (mode & 1) v = __fmul_rn(v, win[i]);
        out[i] = v;
    }
}

// |DFT(x)| of one real line: sign +1 is the reference's ifft (cpu_backend.cpp:
// 634-659: unnormalised exp(+i) transform, magnitude of every output), -1 the
// forward transform; evaluated in double with exact twiddle indices and
// rounded once per component.
__global__ void op_dft_mag_kernel(const float* in, int n, double sign, float* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double re = 0.0, im = 0.0;
    const double w = 6.283185307179586476925286766559 / n;
    for (int j = 0; j < n; ++j) {
        const long long e = ((long long)k * j) % n;
        double s, c;
        sincos(w * (double)e, &s, &c);
        re += (double)in[j] * c;
        im += sign * (double)in[j] * s;
    }
    const float fr = (float)re, fi = (float)im;
    out[k] = __fsqrt_rn(__fadd_rn(__fmul_rn(fr, fr), __fmul_rn(fi, fi)));
}

// The same magnitudes through the chain's own FFT for power-of-two lengths
// 512..8192: one team of N/16 threads runs the Stockham radix-16 passes of the
// fused kernel (fft_twiddle_dft, every output of the last pass) on the line in
// lane a of the packed pairs. For a real line |DFT^-(x)| = |DFT^+(x)| (the two
// transforms are complex conjugates), so both directions use the exp(+i) one.
template <int N>
__global__ void __launch_bounds__(N / 16) op_fft_mag_kernel(const float* in, const float2* tw, float* out) {
    extern __shared__ __align__(16) unsigned char op_smem[];
    float4* exch = reinterpret_cast<float4*>(op_smem);
    constexpr int T = N / 16;
    constexpr int NPASS = Plan<N>::NPASS;
    const int t = threadIdx.x;
    cp v[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) v[s] = cpmake(make_float2(in[t + s * T], 0.0f), make_float2(0.0f, 0.0f));
    fft_twiddle_dft<N, 0, NPASS == 1>(t, v, tw);
    if constexpr (NPASS > 1) {
        fft_store<N, 0>(t, v, exch);
        __syncthreads();
        fft_load<N>(t, exch, v);
        fft_twiddle_dft<N, 1, NPASS == 2>(t, v, tw);
    }
    if constexpr (NPASS > 2) {
        __syncthreads();
        fft_store<N, 1>(t, v, exch);
        __syncthreads();
        fft_load<N>(t, exch, v);
        fft_twiddle_dft<N, 2, NPASS == 3>(t, v, tw);
    }
    if constexpr (NPASS > 3) {
        __syncthreads();
        fft_store<N, 2>(t, v, exch);
        __syncthreads();
        fft_load<N>(t, exch, v);
        fft_twiddle_dft<N, 3, true>(t, v, tw);
    }
    using PI = PassInfo<N, NPASS - 1>;
#pragma unroll
    for (int i = 0; i < PI::D; ++i)
#pragma unroll
        for (int q = 0; q < PI::R; ++q) {
            const cp x = v[i + q * PI::D];
            out[t + i * T + q * (N / PI::R)] =
                __fsqrt_rn(__fadd_rn(__fmul_rn(x.re.x, x.re.x), __fmul_rn(x.im.x, x.im.x)));
        }
}

template <int N>
cudaError_t launch_fft_mag(const float* d_in, const float2* d_tw, float* d_out) {
    constexpr int SMEM = Plan<N>::EXCH_ELEMS * 16;
    cudaError_t e = cudaFuncSetAttribute(op_fft_mag_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    if (e != cudaSuccess) return e;
    op_fft_mag_kernel<N><<<1, N / 16, SMEM>>>(d_in, d_tw, d_out);
    return cudaGetLastError();
}

// getMinimumVarianceMean (cpu_kernels.tpp:402-458), one thread per column,
// the same double accumulation in row order.
__global__ void op_mvm_kernel(const float* in, int width, int height, int segments, float* out) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= width) return;
    const int seg_w = height / segments;
    const float factor = 1.0f / (float)seg_w;
    float min_var = INFINITY, mx = 0.0f, my = 0.0f;
    for (int s = 0; s < segments; ++s) {
        double sx = 0.0, sy = 0.0, sxx = 0.0;
        for (int r = 0; r < seg_w; ++r) {
            const long long idx = ((long long)(s * seg_w + r) * width + col) * 2;
            const double dx = in[idx], dy = in[idx + 1];
            sx += dx;
            sy += dy;
            sxx += __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        }
        const float meanx = (float)(sx * (double)factor), meany = (float)(sy * (double)factor);
        const float var = (float)(__dsub_rn(sxx * (double)factor,
                                            __dadd_rn(__dmul_rn((double)meanx, (double)meanx),
                                                      __dmul_rn((double)meany, (double)meany))));
        if (var < min_var) {
            min_var = var;
            mx = meanx;
            my = meany;
        }
    }
    out[2 * col] = mx;
    out[2 * col + 1] = my;
}

// fixedPatternNoiseRemoval (cpu_backend.cpp:701-733): the mean line is taken
// off the first min(total/2, width) complex values of the flattened data (the
// reference's meanALineSubtraction on the whole buffer), then |z| of all.
__global__ void op_fpn_mag_kernel(const float* in, const float* mean, long long total, long long use, float* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        float re = in[2 * i], im = in[2 * i + 1];
        if (mean && i < use) {
            re = __fsub_rn(re, mean[2 * i]);
            im = __fsub_rn(im, mean[2 * i + 1]);
        }
        out[i] = __fsqrt_rn(__fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im)));
    }
}

// rollingAverageDCRemoval (cpu_kernels.tpp:56-82) per line: float running sum,
// x[i] minus the mean of x[i-(W-1) .. min(i+W, n-1)]. One thread per line.
__global__ void op_rolling_dc_kernel(const float* in, int window, int width, int lines, float* cum, float* out) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= lines) return;
    const float* x = in + (long long)l * width;
    float* c = cum + (long long)l * (width + 1);
    c[0] = 0.0f;
    for (int i = 0; i < width; ++i) c[i + 1] = __fadd_rn(c[i], x[i]);
    for (int i = 0; i < width; ++i) {
        const int start = (i >= window - 1) ? i - (window - 1) : 0;
        const int end = (i + window < width - 1) ? i + window : width - 1;
        const float avg = __fdiv_rn(__fsub_rn(c[end + 1], c[start]), (float)(end - start + 1));
        out[(long long)l * width + i] = __fsub_rn(x[i], avg);
    }
}

// B-scan flip of the chain (cuda_kernels.cu:553-573 semantics): B-scans
// 0, 2, 4, ... that have a successor are mirrored laterally.
__global__ void op_flip_kernel(const float* in, int width, int lines, int bscans, float* out) {
    const long long total = (long long)width * lines * bscans;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / width;
        const int col = (int)(i - row * width);
        const long long b = row / lines;
        long long src = row;
        if ((b & 1) == 0 && b + 1 < bscans) src = b * lines + (lines - 1 - (row - b * lines));
        out[i] = in[src * width + col];
    }
}

// logScaleAndTruncate / linearScaleAndTruncate (cpu_kernels.tpp:301-378) on
// lines of `width` complex values (interleaved), bins [0, width/2) per line;
// auto range per line when min == max (log mode, cpu_backend.cpp:266).
__global__ void op_truncate_kernel(const float* in, int width, long long lines, int log_mode, float gmax,
                                   float gmin, float addend, float mult, float* out) {
    const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (l >= lines) return;
    const int half = width / 2;
    const float* z = in + l * (long long)width * 2;
    float* o = out + l * half;
    float mn = gmin, mx = gmax;
    const bool auto_range = log_mode && gmin == gmax;
    if (auto_range) {
        mn = INFINITY;
        mx = -INFINITY;
    }
    for (int k = 0; k < half; ++k) {
        const float re = z[2 * k], im = z[2 * k + 1];
        const float m2 = __fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im));
        float v;
        if (log_mode) v = __fmul_rn(10.0f, log10f(__fdiv_rn(m2, (float)half)));
        else v = __fdiv_rn(__fsqrt_rn(m2), (float)half);
        o[k] = v;
        if (auto_range) {
            mn = fminf(mn, v);
            mx = fmaxf(mx, v);
        }
    }
    float range = __fsub_rn(mx, mn);
    if (range < 1e-6f) range = 1.0f;
    for (int k = 0; k < half; ++k)
        o[k] = __fmul_rn(mult, __fadd_rn(__fdiv_rn(__fsub_rn(o[k], mn), range), addend));
}

// postProcessBackgroundSubtraction: in[i] - (weight * bg[i % width] + offset).
__global__ void op_bg_kernel(const float* in, const float* bg, float weight, float offset, int width, long long n,
                             float* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = __fsub_rn(in[i], __fadd_rn(__fmul_rn(weight, bg[i % width]), offset));
}

// Device scratch for one synchronous call.
struct Scratch {
    std::vector<void*> p;
    ~Scratch() {
        for (void* q : p) cudaFree(q);
    }
    template <class T>
    cudaError_t alloc(T** out, size_t bytes) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
        if (e == cudaSuccess) p.push_back(q);
        *out = static_cast<T*>(q);
        return e;
    }
    template <class T>
    cudaError_t upload(T** out, const void* host, size_t bytes) {
        cudaError_t e = alloc(out, bytes);
        if (e == cudaSuccess && bytes) e = cudaMemcpy(*out, host, bytes, cudaMemcpyHostToDevice);
        return e;
    }
};

int finish(float* d_out, float* h_out, size_t n) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h_out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? OPE_B200_OK : OPE_B200_E_CUDA;
}

#define OPS_CU(call)                                  \
    do {                                              \
        if ((call) != cudaSuccess) return OPE_B200_E_CUDA; \
    } while (0)

}  // namespace
}  // namespace ope_b200

using namespace ope_b200;

extern "C" {

int ope_b200_op_convert_input(const void* input, int32_t bit_depth, int64_t samples, float* out) {
    if (!input || !out || samples < 1 || bit_depth < 1) return OPE_B200_E_INVALID;
    const size_t esz = bit_depth <= 8 ? 1 : (bit_depth <= 16 ? 2 : 4);
    Scratch s;
    void* d_in;
    float* d_out;
    OPS_CU(s.upload(&d_in, input, esz * samples));
    OPS_CU(s.alloc(&d_out, samples * sizeof(float)));
    op_convert_kernel<<<blocks_for(samples), kThreads>>>(d_in, bit_depth, samples, d_out);
    return finish(d_out, out, samples);
}

int ope_b200_op_klinearization(const float* input, const float* curve, int32_t method, int32_t line_width,
                               int64_t samples, float* out) {
    if (!input || !curve || !out || line_width < 1 || samples < 0 || samples > line_width || method < 0 || method > 2)
        return OPE_B200_E_INVALID;
    Scratch s;
    float *d_in, *d_curve, *d_out;
    OPS_CU(s.upload(&d_in, input, line_width * sizeof(float)));
    OPS_CU(s.upload(&d_curve, curve, line_width * sizeof(float)));
    OPS_CU(s.alloc(&d_out, line_width * sizeof(float)));
    op_klin_kernel<<<blocks_for(line_width), kThreads>>>(d_in, line_width, d_curve, method, line_width, d_out);
    return finish(d_out, out, samples);
}

// mode bit 0: window, bit 1: dispersion (real part).
int ope_b200_op_window_dispersion(const float* input, const float* window, const float* phase_cos_sin, int32_t mode,
                                  int32_t line_width, int64_t samples, float* out) {
    if (!input || !out || line_width < 1 || samples < 0 || samples > line_width || mode < 1 || mode > 3)
        return OPE_B200_E_INVALID;
    if (((mode & 1) && !window) || ((mode & 2) && !phase_cos_sin)) return OPE_B200_E_INVALID;
    Scratch s;
    float *d_in, *d_w = nullptr, *d_cs = nullptr, *d_out;
    OPS_CU(s.upload(&d_in, input, line_width * sizeof(float)));
    if (mode & 1) OPS_CU(s.upload(&d_w, window, line_width * sizeof(float)));
    if (mode & 2) OPS_CU(s.upload(&d_cs, phase_cos_sin, 2 * line_width * sizeof(float)));
    OPS_CU(s.alloc(&d_out, line_width * sizeof(float)));
    op_elementwise_kernel<<<blocks_for(line_width), kThreads>>>(d_in, d_w, d_cs, mode, line_width, d_out);
    return finish(d_out, out, samples);
}

int ope_b200_op_dft_magnitude(const float* input, int32_t line_width, int32_t inverse, float* out) {
    if (!input || !out || line_width < 1) return OPE_B200_E_INVALID;
    Scratch s;
    float *d_in, *d_out;
    OPS_CU(s.upload(&d_in, input, line_width * sizeof(float)));
    OPS_CU(s.alloc(&d_out, line_width * sizeof(float)));
    const int n = line_width;
    if (n >= 512 && n <= 8192 && (n & (n - 1)) == 0) {
        // the chain's FFT (float32, its twiddle table)
        const std::vector<float2> tw = build_twiddles(n);
        float2* d_tw;
        OPS_CU(s.upload(&d_tw, tw.data(), tw.size() * sizeof(float2)));
        cudaError_t e = n == 512    ? launch_fft_mag<512>(d_in, d_tw, d_out)
                        : n == 1024 ? launch_fft_mag<1024>(d_in, d_tw, d_out)
                        : n == 2048 ? launch_fft_mag<2048>(d_in, d_tw, d_out)
                        : n == 4096 ? launch_fft_mag<4096>(d_in, d_tw, d_out)
                                    : launch_fft_mag<8192>(d_in, d_tw, d_out);
        OPS_CU(e);
    } else {
        // any other length: a direct DFT evaluated in double
        op_dft_mag_kernel<<<(n + 127) / 128, 128>>>(d_in, n, inverse ? 1.0 : -1.0, d_out);
    }
    return finish(d_out, out, line_width);
}

int ope_b200_op_min_variance_mean(const float* input, int32_t width, int32_t height, int32_t segments, float* out) {
    if (!input || !out || width < 1 || height < 1 || segments < 1 || height / segments < 1) return OPE_B200_E_INVALID;
    Scratch s;
    float *d_in, *d_out;
    OPS_CU(s.upload(&d_in, input, (size_t)width * height * 2 * sizeof(float)));
    OPS_CU(s.alloc(&d_out, (size_t)width * 2 * sizeof(float)));
    op_mvm_kernel<<<(width + 127) / 128, 128>>>(d_in, width, height, segments, d_out);
    return finish(d_out, out, (size_t)width * 2);
}

int ope_b200_op_fpn_removal(const float* input, const float* mean_line, int32_t line_width, int32_t num_lines,
                            float* out) {
    if (!input || !out || line_width < 1 || num_lines < 1) return OPE_B200_E_INVALID;
    const long long total = (long long)line_width * num_lines;
    const long long use = mean_line ? std::min<long long>(total / 2, line_width) : 0;
    Scratch s;
    float *d_in, *d_mean = nullptr, *d_out;
    OPS_CU(s.upload(&d_in, input, total * 2 * sizeof(float)));
    if (mean_line) OPS_CU(s.upload(&d_mean, mean_line, (size_t)line_width * 2 * sizeof(float)));
    OPS_CU(s.alloc(&d_out, total * sizeof(float)));
    op_fpn_mag_kernel<<<blocks_for(total), kThreads>>>(d_in, d_mean, total, use, d_out);
    return finish(d_out, out, total);
}

int ope_b200_op_rolling_dc_removal(const float* input, int32_t window, int32_t line_width, int32_t num_lines,
                                   float* out) {
    if (!input || !out || window < 1 || line_width < 1 || num_lines < 1) return OPE_B200_E_INVALID;
    const long long total = (long long)line_width * num_lines;
    Scratch s;
    float *d_in, *d_cum, *d_out;
    OPS_CU(s.upload(&d_in, input, total * sizeof(float)));
    OPS_CU(s.alloc(&d_cum, (size_t)(line_width + 1) * num_lines * sizeof(float)));
    OPS_CU(s.alloc(&d_out, total * sizeof(float)));
    op_rolling_dc_kernel<<<(num_lines + 63) / 64, 64>>>(d_in, window, line_width, num_lines, d_cum, d_out);
    return finish(d_out, out, total);
}

int ope_b200_op_bscan_flip(const float* input, int32_t line_width, int32_t lines_per_bscan, int32_t num_bscans,
                           float* out) {
    if (!input || !out || line_width < 1 || lines_per_bscan < 1 || num_bscans < 1) return OPE_B200_E_INVALID;
    const long long total = (long long)line_width * lines_per_bscan * num_bscans;
    Scratch s;
    float *d_in, *d_out;
    OPS_CU(s.upload(&d_in, input, total * sizeof(float)));
    OPS_CU(s.alloc(&d_out, total * sizeof(float)));
    op_flip_kernel<<<blocks_for(total), kThreads>>>(d_in, line_width, lines_per_bscan, num_bscans, d_out);
    return finish(d_out, out, total);
}

int ope_b200_op_sinusoidal_correction(const float* input, const float* curve, int32_t line_width,
                                      int32_t lines_per_bscan, int32_t num_bscans, float* out) {
    if (!input || !out || line_width < 1 || lines_per_bscan < 1 || num_bscans < 1) return OPE_B200_E_INVALID;
    const long long lines = (long long)lines_per_bscan * num_bscans;
    const long long total = lines * line_width;
    Scratch s;
    float *d_in, *d_curve, *d_out;
    OPS_CU(s.upload(&d_in, input, total * sizeof(float)));
    if (curve) {
        OPS_CU(s.upload(&d_curve, curve, lines_per_bscan * sizeof(float)));
    } else {
        OPS_CU(s.alloc(&d_curve, lines_per_bscan * sizeof(float)));
        OPS_CU(sin_curve(d_curve, lines_per_bscan, nullptr));
    }
    OPS_CU(s.alloc(&d_out, total * sizeof(float)));
    OPS_CU(sin_correct(d_out, d_in, d_curve, line_width, lines_per_bscan, lines, nullptr, nullptr));
    return finish(d_out, out, total);
}

int ope_b200_op_truncate(const float* input, int32_t log_scaling, float grayscale_max, float grayscale_min,
                         float addend, float multiplicator, int32_t line_width, int64_t num_lines, float* out) {
    if (!input || !out || line_width < 2 || num_lines < 1) return OPE_B200_E_INVALID;
    Scratch s;
    float *d_in, *d_out;
    OPS_CU(s.upload(&d_in, input, (size_t)line_width * 2 * num_lines * sizeof(float)));
    OPS_CU(s.alloc(&d_out, (size_t)(line_width / 2) * num_lines * sizeof(float)));
    op_truncate_kernel<<<(unsigned)((num_lines + 63) / 64), 64>>>(d_in, line_width, num_lines, log_scaling ? 1 : 0,
                                                                  grayscale_max, grayscale_min, addend,
                                                                  multiplicator, d_out);
    return finish(d_out, out, (size_t)(line_width / 2) * num_lines);
}

int ope_b200_op_background_subtraction(const float* input, const float* background_line, float weight,
                                       float offset, int32_t line_width, int64_t samples, float* out) {
    if (!input || !background_line || !out || line_width < 1 || samples < 0) return OPE_B200_E_INVALID;
    Scratch s;
    float *d_in, *d_bg, *d_out;
    OPS_CU(s.upload(&d_in, input, samples * sizeof(float)));
    OPS_CU(s.upload(&d_bg, background_line, line_width * sizeof(float)));
    OPS_CU(s.alloc(&d_out, samples * sizeof(float)));
    op_bg_kernel<<<blocks_for(samples), kThreads>>>(d_in, d_bg, weight, offset, line_width, samples, d_out);
    return finish(d_out, out, samples);
}

}  // extern "C"
