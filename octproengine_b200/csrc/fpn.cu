// Fixed-pattern-noise determination: reduction, minimum-variance selection
// and host-side state machine (see fpn.h).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fpn.h"

namespace ope_b200 {

// acc[s][i] += sum over bx of partial[s][bx][i], i over (n/2)*3 values, in bx order.
__global__ void fpn_reduce_kernel(const double* __restrict__ partial, double* __restrict__ acc, int gx, int per_seg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (i >= per_seg) return;
    const double* p = partial + (long long)s * gx * per_seg + i;
    double sum = 0.0;
    for (int b = 0; b < gx; ++b) sum += p[(long long)b * per_seg];
    acc[(long long)s * per_seg + i] += sum;
}

// Minimum-variance segment mean per bin, following getMinimumVarianceMean
// (cpu_kernels.tpp:414-455): float factor 1/seg_w, double moments, float
// mean and variance, first strict minimum wins. Explicit _rn operations keep
// the double arithmetic uncontracted like the reference's.
__global__ void fpn_finalize_kernel(const double* __restrict__ acc, float2* __restrict__ profile, int half,
                                    long long seg_w) {
    const int bin = blockIdx.x * blockDim.x + threadIdx.x;
    if (bin >= half) return;
    const float factor = __fdiv_rn(1.0f, (float)seg_w);
    const double fd = (double)factor;
    float min_var = INFINITY, mx = 0.0f, my = 0.0f;
    for (int s = 0; s < FPN_SEGMENTS; ++s) {
        const double* a = acc + ((long long)s * half + bin) * 3;
        const float mean_x = (float)__dmul_rn(a[0], fd);
        const float mean_y = (float)__dmul_rn(a[1], fd);
        const double m2 = __dadd_rn(__dmul_rn((double)mean_x, (double)mean_x), __dmul_rn((double)mean_y, (double)mean_y));
        const float var = (float)__dsub_rn(__dmul_rn(a[2], fd), m2);
        if (var < min_var) {
            min_var = var;
            mx = mean_x;
            my = mean_y;
        }
    }
    profile[bin] = make_float2(mx, my);
}

cudaError_t fpn_init(FpnState& st, int n) {
    st.n = n;
    const size_t half = n / 2;
    cudaError_t e = cudaMalloc(&st.d_acc, FPN_SEGMENTS * half * 3 * sizeof(double));
    if (e != cudaSuccess) return e;
    e = cudaMalloc(&st.d_profile, half * sizeof(float2));
    if (e != cudaSuccess) return e;
    return cudaMemset(st.d_profile, 0, half * sizeof(float2));
}

void fpn_free(FpnState& st) {
    cudaFree(st.d_acc);
    cudaFree(st.d_partial);
    cudaFree(st.d_profile);
    st.d_acc = st.d_partial = nullptr;
    st.d_profile = nullptr;
}

static int cuerr(std::string* err, cudaError_t e, const char* what) {
    if (err) *err = std::string(what) + ": " + cudaGetErrorString(e);
    return OPE_B200_E_CUDA;
}

int fpn_process_frame(FpnState& st, const ope_b200_config& cfg, int in_kind, int interp, const ChainArgs& a,
                      cudaStream_t s, std::string* err) {
    const long long required = (long long)cfg.fpn_bscan_count * cfg.ascans_per_bscan;
    if (!st.active) {
        if (!(st.requested || cfg.fpn_continuous)) return OPE_B200_OK;
        st.active = true;
        st.requested = false;
        st.acc_rows = 0;
        cudaError_t e = cudaMemsetAsync(st.d_acc, 0, FPN_SEGMENTS * (size_t)(st.n / 2) * 3 * sizeof(double), s);
        if (e != cudaSuccess) return cuerr(err, e, "fpn accumulator reset");
    }
    const long long seg_w = required / FPN_SEGMENTS;
    if (seg_w < 1) {
        st.active = false;
        if (err) *err = "fixed-pattern noise determination needs at least 8 A-scans";
        return OPE_B200_E_INVALID;
    }
    const long long use = std::min<long long>(a.m, required - st.acc_rows);
    const long long pairs_per_seg = (seg_w + 1) / 2;
    const int gx = (int)std::max<long long>(1, std::min<long long>(64, (pairs_per_seg + 3) / 4));
    const int half = st.n / 2;
    const size_t need = (size_t)FPN_SEGMENTS * gx * half * 3;
    if (need > st.partial_cap) {
        cudaFree(st.d_partial);
        st.d_partial = nullptr;
        st.partial_cap = 0;
        cudaError_t e = cudaMalloc(&st.d_partial, need * sizeof(double));
        if (e != cudaSuccess) return cuerr(err, e, "fpn scratch allocation");
        st.partial_cap = need;
    }
    cudaError_t e = launch_fpn_stats(st.n, in_kind, interp, a, st.acc_rows, use, seg_w, gx, st.d_partial, s);
    if (e != cudaSuccess) return cuerr(err, e, "fpn statistics launch");
    const int per_seg = half * 3;
    fpn_reduce_kernel<<<dim3((per_seg + 255) / 256, FPN_SEGMENTS), 256, 0, s>>>(st.d_partial, st.d_acc, gx, per_seg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuerr(err, e, "fpn reduce launch");
    st.acc_rows += use;
    if (st.acc_rows >= required) {
        fpn_finalize_kernel<<<(half + 255) / 256, 256, 0, s>>>(st.d_acc, st.d_profile, half, seg_w);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuerr(err, e, "fpn finalize launch");
        st.valid = true;
        st.host_dirty = true;
        st.active = false;
    }
    return OPE_B200_OK;
}

int fpn_set_profile(FpnState& st, const float* p, size_t pairs, cudaStream_t s, std::string* err) {
    const size_t half = st.n / 2;
    // setFixedPatternNoiseProfile stores what it is given; meanALineSubtraction
    // then uses min(N/2, pairs) bins (cpu_kernels.tpp:468-478).
    std::vector<float> prof(2 * half, 0.0f);
    const size_t use = std::min(pairs, half);
    if (use) std::memcpy(prof.data(), p, use * 2 * sizeof(float));
    // frames in flight on any stream may read the profile: drain the device
    (void)s;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuerr(err, e, "fpn profile sync");
    e = cudaMemcpy(st.d_profile, prof.data(), half * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuerr(err, e, "fpn profile upload");
    st.host_profile.assign(p, p + pairs * 2);
    st.host_dirty = false;
    st.valid = pairs > 0;
    return OPE_B200_OK;
}

int fpn_get_profile(FpnState& st, float* out, size_t cap_pairs, size_t* pairs, std::string* err) {
    if (st.host_dirty) {
        const size_t half = st.n / 2;
        st.host_profile.assign(2 * half, 0.0f);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return cuerr(err, e, "fpn profile sync");
        e = cudaMemcpy(st.host_profile.data(), st.d_profile, half * sizeof(float2), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuerr(err, e, "fpn profile download");
        st.host_dirty = false;
    }
    const size_t have = st.valid ? st.host_profile.size() / 2 : 0;
    if (pairs) *pairs = have;
    if (out) std::memcpy(out, st.host_profile.data(), std::min(have, cap_pairs) * 2 * sizeof(float));
    return OPE_B200_OK;
}

cudaError_t launch_fpn_reduce(const double* partial, double* acc, int gx, int half, cudaStream_t s) {
    const int per_seg = half * 3;
    fpn_reduce_kernel<<<dim3((per_seg + 255) / 256, FPN_SEGMENTS), 256, 0, s>>>(partial, acc, gx, per_seg);
    return cudaGetLastError();
}

cudaError_t launch_fpn_finalize(const double* acc, float2* profile, int half, long long seg_w, cudaStream_t s) {
    fpn_finalize_kernel<<<(half + 255) / 256, 256, 0, s>>>(acc, profile, half, seg_w);
    return cudaGetLastError();
}

cudaError_t launch_fpn_stats(int n, int in_kind, int interp, const ChainArgs& a, long long g0, long long rows,
                             long long seg_w, int gx, double* partial, cudaStream_t s) {
    switch (n) {
        case 512: return launch_fpn_stats_n512(in_kind, interp, a, g0, rows, seg_w, gx, partial, s);
        case 1024: return launch_fpn_stats_n1024(in_kind, interp, a, g0, rows, seg_w, gx, partial, s);
        case 2048: return launch_fpn_stats_n2048(in_kind, interp, a, g0, rows, seg_w, gx, partial, s);
        case 4096: return launch_fpn_stats_n4096(in_kind, interp, a, g0, rows, seg_w, gx, partial, s);
        case 8192: return launch_fpn_stats_n8192(in_kind, interp, a, g0, rows, seg_w, gx, partial, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ope_b200
