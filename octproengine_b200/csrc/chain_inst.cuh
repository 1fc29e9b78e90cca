// Instantiates the fused chain kernels for one FFT length OPE_CHAIN_N.
// Included by chain_n<N>.cu; compiled once per length so the variants build
// in parallel.
#include <mutex>

#include "chain_device.cuh"
#include "chain_launch.h"
#include "fpn.h"

#ifndef OPE_CHAIN_N
#error "define OPE_CHAIN_N"
#endif

namespace ope_b200 {
namespace {

template <int N, int DT, int INTERP>
cudaError_t launch_variant(const ChainArgs& a, cudaStream_t stream, int max_ctas, LaunchInfo* info) {
    constexpr int SMEM = Layout<N, DT>::TOTAL;
    constexpr int BLOCK = N / 16;
    auto kern = chain_kernel<N, DT, INTERP>;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    // per-device attribute set-up and occupancy, cached
    static std::mutex mu;
    static int per_sm[64] = {0};
    static int sms[64] = {0};
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (per_sm[dev] == 0) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
            if (e != cudaSuccess) return e;
            int occ = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, BLOCK, SMEM);
            if (e != cudaSuccess) return e;
            int nsm = 0;
            e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
            if (occ < 1) return cudaErrorInvalidConfiguration;
            sms[dev] = nsm;
            per_sm[dev] = occ;
        }
    }
    const long long npairs = (a.m + 1) / 2;
    long long grid = (long long)per_sm[dev] * sms[dev];
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    if (grid > npairs) grid = npairs;
    if (grid < 1) grid = 1;
    if (info) {
        info->grid = (int)grid;
        info->block = BLOCK;
        info->smem = SMEM;
        info->blocks_per_sm = per_sm[dev];
    }
    kern<<<(unsigned)grid, BLOCK, SMEM, stream>>>(a);
    return cudaGetLastError();
}

template <int N, int DT>
cudaError_t dispatch_interp(int interp, const ChainArgs& a, cudaStream_t s, int max_ctas, LaunchInfo* info) {
    switch (interp) {
        case INTERP_NONE: return launch_variant<N, DT, INTERP_NONE>(a, s, max_ctas, info);
        case INTERP_LINEAR: return launch_variant<N, DT, INTERP_LINEAR>(a, s, max_ctas, info);
        case INTERP_CUBIC: return launch_variant<N, DT, INTERP_CUBIC>(a, s, max_ctas, info);
        case INTERP_LANCZOS: return launch_variant<N, DT, INTERP_LANCZOS>(a, s, max_ctas, info);
        default: return cudaErrorInvalidValue;
    }
}

template <int N, int DT, int INTERP>
cudaError_t launch_fpn_variant(const ChainArgs& a, long long g0, long long rows, long long seg_w, int gx,
                               double* partial, cudaStream_t s) {
    constexpr int SMEM = Layout<N, DT>::TOTAL;
    auto kern = fpn_stats_kernel<N, DT, INTERP>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    if (e != cudaSuccess) return e;
    dim3 grid(gx, FPN_SEGMENTS);
    kern<<<grid, N / 16, SMEM, s>>>(a, g0, rows, seg_w, partial);
    return cudaGetLastError();
}

template <int N, int DT>
cudaError_t fpn_dispatch_interp(int interp, const ChainArgs& a, long long g0, long long rows, long long seg_w,
                                int gx, double* partial, cudaStream_t s) {
    switch (interp) {
        case INTERP_NONE: return launch_fpn_variant<N, DT, INTERP_NONE>(a, g0, rows, seg_w, gx, partial, s);
        case INTERP_LINEAR: return launch_fpn_variant<N, DT, INTERP_LINEAR>(a, g0, rows, seg_w, gx, partial, s);
        case INTERP_CUBIC: return launch_fpn_variant<N, DT, INTERP_CUBIC>(a, g0, rows, seg_w, gx, partial, s);
        case INTERP_LANCZOS: return launch_fpn_variant<N, DT, INTERP_LANCZOS>(a, g0, rows, seg_w, gx, partial, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

#define OPE_B200_CAT2(a, b) a##b
#define OPE_B200_CAT(a, b) OPE_B200_CAT2(a, b)

cudaError_t OPE_B200_CAT(launch_chain_n, OPE_CHAIN_N)(int in_kind, int interp, const ChainArgs& a,
                                                      cudaStream_t stream, int max_ctas, LaunchInfo* info) {
    constexpr int N = OPE_CHAIN_N;
    switch (in_kind) {
        case IN_U8: return dispatch_interp<N, IN_U8>(interp, a, stream, max_ctas, info);
        case IN_U16: return dispatch_interp<N, IN_U16>(interp, a, stream, max_ctas, info);
        case IN_U32: return dispatch_interp<N, IN_U32>(interp, a, stream, max_ctas, info);
        case IN_F32: return dispatch_interp<N, IN_F32>(interp, a, stream, max_ctas, info);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t OPE_B200_CAT(launch_fpn_stats_n, OPE_CHAIN_N)(int in_kind, int interp, const ChainArgs& a, long long g0,
                                                          long long rows, long long seg_w, int gx, double* partial,
                                                          cudaStream_t s) {
    constexpr int N = OPE_CHAIN_N;
    switch (in_kind) {
        case IN_U8: return fpn_dispatch_interp<N, IN_U8>(interp, a, g0, rows, seg_w, gx, partial, s);
        case IN_U16: return fpn_dispatch_interp<N, IN_U16>(interp, a, g0, rows, seg_w, gx, partial, s);
        case IN_U32: return fpn_dispatch_interp<N, IN_U32>(interp, a, g0, rows, seg_w, gx, partial, s);
        case IN_F32: return fpn_dispatch_interp<N, IN_F32>(interp, a, g0, rows, seg_w, gx, partial, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ope_b200
