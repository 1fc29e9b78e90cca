// C ABI of the differentiable chain (autofocus): device-built tables,
// entropy forward and the hand-written adjoint. See autofocus.cuh for the
// mathematics; the entry points are declared in include/ope_b200.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/ope_b200.h"
#include "af_launch.h"
#include "autofocus.cuh"
#include "tables.h"

using namespace ope_b200;

namespace ope_b200 {

__device__ __forceinline__ int af_trunc(float v) {
    if (!(v == v)) return 0;
    if (v > 1.0e8f) return 100000000;
    if (v < -1.0e8f) return -100000000;
    return (int)v;
}

__device__ __forceinline__ void af_tables(int j, int n, int interp, const float* __restrict__ params,
                                          const float* __restrict__ window, int2* lin, int2* cub, int* lzb,
                                          float* rmask, float2* wph) {
    if (j >= n) return;
    // resampling position (processorconfiguration.cpp:438-459)
    const float s1 = (float)n - 1.0f;
    const float c0 = params[4];
    const float c1 = __fdiv_rn(params[5], s1);
    const float c2 = __fdiv_rn(params[6], __fmul_rn(s1, s1));
    const float c3 = __fdiv_rn(params[7], __fmul_rn(__fmul_rn(s1, s1), s1));
    const float x = (float)j;
    const float v = __fadd_rn(c0, __fmul_rn(x, __fadd_rn(c1, __fmul_rn(x, __fadd_rn(c2, __fmul_rn(x, c3))))));
    const float lo = 7.0f, hi = (float)(n - 9);
    const bool inside = (v >= lo) && (v <= hi);
    const float nx = inside ? v : ((v > hi) ? hi : lo);  // NaN -> lo
    rmask[j] = inside ? 1.0f : 0.0f;
    auto cl = [n](int q) { return q > n - 1 ? n - 1 : (q < -SPEC_PAD ? -SPEC_PAD : q); };
    if (interp == INTERP_LINEAR) {
        const int n1 = cl(af_trunc(nx));
        lin[j] = make_int2(n1 + SPEC_PAD, __float_as_int(__fsub_rn(nx, (float)n1)));
    } else if (interp == INTERP_CUBIC) {
        const int i1 = af_trunc(nx);
        const int n1r = cl(i1);
        const int q0 = cl(abs(i1 - 1)) + SPEC_PAD, q1 = n1r + SPEC_PAD;
        const float pos = __fsub_rn(nx, (float)n1r);
        cub[j] = make_int2(q0 | (q1 << 16), __float_as_int(pos));
    } else if (interp == INTERP_LANCZOS) {
        const int n0 = af_trunc(nx);
        int b = n0 < -9 ? -9 : (n0 > n + 7 ? n + 7 : n0);
        lzb[j] = b - 7 + SPEC_PAD;
        // the 16 tap weights (and derivatives) come from af_lanczos
    }
    // dispersion phase (processorconfiguration.cpp:461-482), window x (cos, sin)
    const float d0 = params[0];
    const float d1 = __fdiv_rn(params[1], s1);
    const float d2 = __fdiv_rn(params[2], __fmul_rn(s1, s1));
    const float d3 = __fdiv_rn(params[3], __fmul_rn(__fmul_rn(s1, s1), s1));
    const float ph = __fadd_rn(d0, __fmul_rn(x, __fadd_rn(d1, __fmul_rn(x, __fadd_rn(d2, __fmul_rn(x, d3))))));
    float sn, cs;
    sincosf(ph, &sn, &cs);
    const double w = window ? (double)window[j] : 1.0;
    const float wc = (float)(w * (double)cs), ws = (float)(w * (double)sn);
    wph[j] = make_float2(wc, ws);
}

// Lanczos-8 tap weights of every output sample, one thread per (tap, sample);
// derivative weights only when the adjoint needs them.
__device__ __forceinline__ void af_lanczos(int i, int n, const float* __restrict__ params, float* lzw,
                                           float* lzdw) {
    if (i >= 16 * n) return;
    const int k = i / n, j = i - k * n;
    const float s1 = (float)n - 1.0f;
    const float c0 = params[4];
    const float c1 = __fdiv_rn(params[5], s1);
    const float c2 = __fdiv_rn(params[6], __fmul_rn(s1, s1));
    const float c3 = __fdiv_rn(params[7], __fmul_rn(__fmul_rn(s1, s1), s1));
    const float x = (float)j;
    const float v = __fadd_rn(c0, __fmul_rn(x, __fadd_rn(c1, __fmul_rn(x, __fadd_rn(c2, __fmul_rn(x, c3))))));
    const float lo = 7.0f, hi = (float)(n - 9);
    const float nx = (v >= lo && v <= hi) ? v : ((v > hi) ? hi : lo);
    int idx = af_trunc(nx) - 7 + k;
    idx = idx < 0 ? 0 : (idx >= n ? n - 1 : idx);
    const float d = __fsub_rn(nx, (float)idx);
    lzw[i] = af_lanczos8(d);
    if (lzdw) lzdw[i] = af_lanczos8_deriv(d);
}

// Every table of one evaluation in one launch: blocks [0, tb) build the
// per-sample tables, the blocks after them (Lanczos-8 only) the 16 tap
// weights per sample.
__global__ void af_prepare_kernel(int n, int interp, int tb, const float* __restrict__ params,
                                  const float* __restrict__ window, int2* lin, int2* cub, int* lzb, float* lzw,
                                  float* lzdw, float* rmask, float2* wph) {
    if ((int)blockIdx.x < tb)
        af_tables(blockIdx.x * blockDim.x + threadIdx.x, n, interp, params, window, lin, cub, lzb, rmask, wph);
    else
        af_lanczos(((int)blockIdx.x - tb) * blockDim.x + threadIdx.x, n, params, lzw, lzdw);
}

// Deterministic block sum of `width` interleaved values per record over
// `nrec` records: thread i sums records i, i + 256, ... in order, then a fixed
// shared-memory tree. One block of 256 threads.
template <int W>
__device__ __forceinline__ void af_block_sum(const double* partial, int nrec, double* out) {
    __shared__ double sh[W][256];
    const int t = threadIdx.x;
    double acc[W];
#pragma unroll
    for (int k = 0; k < W; ++k) acc[k] = 0.0;
    for (int b = t; b < nrec; b += 256)
#pragma unroll
        for (int k = 0; k < W; ++k) acc[k] += partial[W * b + k];
#pragma unroll
    for (int k = 0; k < W; ++k) sh[k][t] = acc[k];
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (t < h)
#pragma unroll
            for (int k = 0; k < W; ++k) sh[k][t] += sh[k][t + h];
        __syncthreads();
    }
    if (t < W) out[t] = sh[t][0];
}

// H = ln S - (sum I ln I)/S from the per-CTA sums.
__global__ void __launch_bounds__(256) af_entropy_finalize(const double* partial, int nblocks, double* hs) {
    __shared__ double r[2];
    af_block_sum<2>(partial, nblocks, r);
    __syncthreads();
    if (threadIdx.x == 0) {
        const double s = r[0], e = r[1];
        hs[0] = (s > 0.0) ? log(s) - e / s : 0.0;
        hs[1] = s;
    }
}

__global__ void __launch_bounds__(256) af_grad_finalize(const double* partial, int nblocks, float* grad) {
    __shared__ double r[AF_NPARAM];
    af_block_sum<AF_NPARAM>(partial, nblocks, r);
    __syncthreads();
    if (threadIdx.x < AF_NPARAM) grad[threadIdx.x] = (float)r[threadIdx.x];
}

}  // namespace ope_b200

struct ope_b200_af {
    int n = 0;
    int in_kind = 0;
    int interp = INTERP_LINEAR;
    int device = 0;
    float* window = nullptr;
    float2* tw = nullptr;
    float2* dc_zero = nullptr;
    int2* lin = nullptr;
    int2* cub = nullptr;
    int* lzb = nullptr;
    float* lzw = nullptr;
    float* lzdw = nullptr;
    float* rmask = nullptr;
    float2* wph = nullptr;
    double* partial = nullptr;
    int cap = 0;
    const float* tables_params = nullptr;  // parameter pointer the device tables were last built from
    int bitshift = 0;  // 8/16-bit samples >> 4 before the chain (DataParameters::bitshift)
    std::string err;
};

namespace {

int af_fail(ope_b200_af* a, int code, const std::string& msg) {
    if (a) a->err = msg;
    return code;
}

int af_cuda(ope_b200_af* a, cudaError_t e, const char* what) {
    return af_fail(a, OPE_B200_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define AF_CU(obj, call)                                         \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return af_cuda(obj, e_, #call);   \
    } while (0)

void af_free(ope_b200_af* a) {
    cudaFree(a->window);
    cudaFree(a->tw);
    cudaFree(a->dc_zero);
    cudaFree(a->lin);
    cudaFree(a->cub);
    cudaFree(a->lzb);
    cudaFree(a->lzw);
    cudaFree(a->lzdw);
    cudaFree(a->rmask);
    cudaFree(a->wph);
    cudaFree(a->partial);
}

cudaError_t af_launch(bool backward, ope_b200_af* o, const AfArgs& args, cudaStream_t s, int* grid) {
    switch (o->n) {
        case 1024: return af_launch_n1024(backward, o->in_kind, o->interp, args, s, o->cap, grid);
        case 2048: return af_launch_n2048(backward, o->in_kind, o->interp, args, s, o->cap, grid);
        case 4096: return af_launch_n4096(backward, o->in_kind, o->interp, args, s, o->cap, grid);
        default: return cudaErrorInvalidValue;
    }
}

// build_tables: false reuses the tables of the previous call (same parameters,
// stream-ordered after it).
int af_prepare(ope_b200_af* o, const void* d_in, int64_t num_ascans, const float* d_params, cudaStream_t s,
               bool backward, AfArgs* args, bool build_tables = true) {
    if (!d_in || !d_params) return af_fail(o, OPE_B200_E_INVALID, "null input or parameter pointer");
    if (num_ascans < 1) return af_fail(o, OPE_B200_E_INVALID, "num_ascans must be >= 1");
    if ((reinterpret_cast<uintptr_t>(d_in) & 15u) != 0)
        return af_fail(o, OPE_B200_E_INVALID, "input must be 16-byte aligned");
    AF_CU(o, cudaSetDevice(o->device));
    if (build_tables) {
        const int threads = 256;
        const int tb = (o->n + threads - 1) / threads;
        const int lb = o->interp == INTERP_LANCZOS ? (16 * o->n + threads - 1) / threads : 0;
        af_prepare_kernel<<<tb + lb, threads, 0, s>>>(o->n, o->interp, tb, d_params, o->window, o->lin, o->cub,
                                                      o->lzb, o->lzw, backward ? o->lzdw : nullptr, o->rmask,
                                                      o->wph);
        AF_CU(o, cudaGetLastError());
        o->tables_params = d_params;
    }
    AfArgs a{};
    a.c.in = d_in;
    a.c.m = num_ascans;
    a.c.tw = o->tw;
    a.c.lin = o->lin;
    a.c.cub = o->cub;
    a.c.lz_base = o->lzb;
    a.c.lz_w = o->lzw;
    a.c.wph = o->wph;
    a.c.dc_resp = o->dc_zero;  // integer-mean split, nothing added back
    a.c.timeout_ns = 2000000000ull;
    a.c.neg_zero = -0.0f;
    a.c.bitshift = o->bitshift;
    a.lz_dw = o->lzdw;
    a.rmask = o->rmask;
    a.partial = o->partial;
    *args = a;
    return OPE_B200_OK;
}

}  // namespace

// A few bytes moved by one warp pair's loads and stores. Between page-locked
// host memory and the device this crosses the link as ordinary memory traffic,
// so it does not queue behind bulk copies waiting on the copy engines (a fit's
// parameter upload and result download while frames stream in and out).
constexpr int AF_SMALL_COPY_MAX = 4096;

__global__ void af_small_copy_kernel(unsigned char* dst, const unsigned char* src, int bytes) {
    for (int i = threadIdx.x; i < bytes; i += blockDim.x) dst[i] = src[i];
}

extern "C" {

int ope_b200_af_set_bitshift(ope_b200_af* af, int32_t on) {
    if (!af) return OPE_B200_E_INVALID;
    af->bitshift = (on && (af->in_kind == IN_U8 || af->in_kind == IN_U16)) ? 1 : 0;
    return OPE_B200_OK;
}

int ope_b200_af_create(int32_t n, int32_t input_dtype, int32_t interpolation, const float* window, int32_t device,
                       ope_b200_af** out) {
    if (!out) return OPE_B200_E_INVALID;
    *out = nullptr;
    auto* o = new ope_b200_af();
    if (n != 1024 && n != 2048 && n != 4096) {
        delete o;
        return OPE_B200_E_UNSUPPORTED;
    }
    switch (input_dtype) {
        case 1: o->in_kind = IN_U8; break;   // ope::DataType::UINT8
        case 2: o->in_kind = IN_U16; break;  // UINT16
        case 9: o->in_kind = IN_F32; break;  // FLOAT32 (read as float)
        default: delete o; return OPE_B200_E_UNSUPPORTED;
    }
    if (interpolation < 0 || interpolation > 2) {
        delete o;
        return OPE_B200_E_INVALID;
    }
    o->n = n;
    o->interp = interpolation + 1;  // ope::InterpolationMethod -> kernel enum
    o->device = device;
    auto bail = [&](cudaError_t e) {
        af_free(o);
        delete o;
        (void)e;
        return OPE_B200_E_CUDA;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(e);
    int nsm = 0;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return bail(e);
    o->cap = nsm * 8;
    const size_t nn = static_cast<size_t>(n);
    if ((e = cudaMalloc(&o->window, nn * 4)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->tw, nn * 8)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->dc_zero, nn / 2 * 8)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->lin, nn * 8)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->cub, nn * 8)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->lzb, nn * 4)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->lzw, nn * 16 * 4)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->lzdw, nn * 16 * 4)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->rmask, nn * 4)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->wph, nn * 8)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&o->partial, static_cast<size_t>(o->cap) * AF_NPARAM * 8)) != cudaSuccess) return bail(e);
    std::vector<float> w(nn, 1.0f);
    if (window) w.assign(window, window + nn);
    const std::vector<float2> tw = build_twiddles(n);
    if ((e = cudaMemcpy(o->window, w.data(), nn * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e);
    if ((e = cudaMemcpy(o->tw, tw.data(), nn * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e);
    if ((e = cudaMemset(o->dc_zero, 0, nn / 2 * 8)) != cudaSuccess) return bail(e);
    *out = o;
    return OPE_B200_OK;
}

void ope_b200_af_destroy(ope_b200_af* o) {
    if (!o) return;
    cudaSetDevice(o->device);
    cudaDeviceSynchronize();
    af_free(o);
    delete o;
}

const char* ope_b200_af_last_error(const ope_b200_af* o) { return o ? o->err.c_str() : "null autofocus handle"; }

int ope_b200_af_forward(ope_b200_af* o, const void* d_in, int64_t num_ascans, const float* d_params,
                        int32_t output_mode, float* d_out, double* d_hs, void* stream) {
    if (!o) return OPE_B200_E_INVALID;
    if (!d_out && !d_hs) return af_fail(o, OPE_B200_E_INVALID, "nothing to compute: d_out and d_hs are both null");
    if (d_out && output_mode != AF_OUT_INTENSITY && output_mode != AF_OUT_DB)
        return af_fail(o, OPE_B200_E_INVALID, "output_mode must be 1 (intensity) or 2 (dB)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    AfArgs a;
    int rc = af_prepare(o, d_in, num_ascans, d_params, s, false, &a);
    if (rc != OPE_B200_OK) return rc;
    a.out = d_out;
    a.out_mode = d_out ? output_mode : AF_OUT_NONE;
    int grid = 0;
    AF_CU(o, af_launch(false, o, a, s, &grid));
    if (d_hs) {
        af_entropy_finalize<<<1, 256, 0, s>>>(o->partial, grid, d_hs);
        AF_CU(o, cudaGetLastError());
    }
    return OPE_B200_OK;
}

static int af_backward_impl(ope_b200_af* o, const void* d_in, int64_t num_ascans, const float* d_params,
                            int32_t output_mode, const float* d_grad_out, const double* d_hs, float* d_grad_params,
                            void* stream, bool disp_only) {
    if (!o) return OPE_B200_E_INVALID;
    if (!d_grad_params) return af_fail(o, OPE_B200_E_INVALID, "null gradient output");
    if (!d_grad_out && !d_hs)
        return af_fail(o, OPE_B200_E_INVALID, "need d_grad_out (image gradient) or d_hs (entropy objective)");
    if (d_grad_out && output_mode != AF_OUT_INTENSITY && output_mode != AF_OUT_DB)
        return af_fail(o, OPE_B200_E_INVALID, "output_mode must be 1 (intensity) or 2 (dB)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    AfArgs a;
    // the dispersion-only adjoint needs no derivative tables: it reuses the
    // forward's when they were built from the same parameter pointer
    const bool reuse = disp_only && o->tables_params == d_params;
    int rc = af_prepare(o, d_in, num_ascans, d_params, s, !disp_only, &a, !reuse);
    if (rc != OPE_B200_OK) return rc;
    a.grad_out = d_grad_out;
    a.out_mode = d_grad_out ? output_mode : AF_OUT_NONE;
    a.hs = d_hs;
    a.disp_only = disp_only ? 1 : 0;
    int grid = 0;
    AF_CU(o, af_launch(true, o, a, s, &grid));
    af_grad_finalize<<<1, 256, 0, s>>>(o->partial, grid, d_grad_params);
    AF_CU(o, cudaGetLastError());
    return OPE_B200_OK;
}

int ope_b200_af_backward(ope_b200_af* o, const void* d_in, int64_t num_ascans, const float* d_params,
                         int32_t output_mode, const float* d_grad_out, const double* d_hs, float* d_grad_params,
                         void* stream) {
    return af_backward_impl(o, d_in, num_ascans, d_params, output_mode, d_grad_out, d_hs, d_grad_params, stream,
                            false);
}

int ope_b200_af_backward_dispersion(ope_b200_af* o, const void* d_in, int64_t num_ascans, const float* d_params,
                                    int32_t output_mode, const float* d_grad_out, const double* d_hs,
                                    float* d_grad_params, void* stream) {
    return af_backward_impl(o, d_in, num_ascans, d_params, output_mode, d_grad_out, d_hs, d_grad_params, stream,
                            true);
}

int ope_b200_af_kernel_accessible(const void* ptr) {
    if (!ptr) return 0;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) return 1;
    // page-locked host memory: usable in kernels at the same address (unified addressing)
    return at.type == cudaMemoryTypeHost && at.devicePointer == ptr ? 1 : 0;
}

int ope_b200_af_small_copy(void* dst, const void* src, int32_t bytes, void* stream) {
    if (!dst || !src || bytes < 0 || bytes > AF_SMALL_COPY_MAX) return OPE_B200_E_INVALID;
    if (bytes == 0) return OPE_B200_OK;
    af_small_copy_kernel<<<1, 64, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<unsigned char*>(dst), static_cast<const unsigned char*>(src), bytes);
    return cudaGetLastError() == cudaSuccess ? OPE_B200_OK : OPE_B200_E_CUDA;
}

}  // extern "C"
