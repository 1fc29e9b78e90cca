// Instantiates the autofocus forward/adjoint kernels for one FFT length
// OPE_AF_N (input types uint16 / float32 / uint8, interpolation linear /
// cubic / Lanczos-8). Included by af_n<N>.cu.
#include <mutex>

#include "af_launch.h"
#include "autofocus.cuh"

#ifndef OPE_AF_N
#error "define OPE_AF_N"
#endif

namespace ope_b200 {
namespace {

struct Occ {
    std::mutex mu;
    int per_sm[64] = {0};
    int sms[64] = {0};
};

template <class K>
cudaError_t occupancy(K kern, int block, int smem, Occ& o, int* per_sm, int* sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(o.mu);
    if (o.per_sm[dev] == 0) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        int occ = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, smem);
        if (e != cudaSuccess) return e;
        int nsm = 0;
        e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (occ < 1) return cudaErrorInvalidConfiguration;
        o.per_sm[dev] = occ;
        o.sms[dev] = nsm;
    }
    *per_sm = o.per_sm[dev];
    *sms = o.sms[dev];
    return cudaSuccess;
}

long long grid_for(long long npairs, int per_sm, int sms, int cap) {
    long long g = (long long)per_sm * sms;
    if (g > cap) g = cap;
    if (g > npairs) g = npairs;
    return g < 1 ? 1 : g;
}

template <int N, int DT, int INTERP>
cudaError_t fwd_variant(const AfArgs& a, cudaStream_t s, int cap, int* grid) {
    constexpr int SMEM = Layout<N, DT>::TOTAL;
    static Occ o;
    int per_sm = 0, sms = 0;
    auto kern = af_forward_kernel<N, DT, INTERP>;
    cudaError_t e = occupancy(kern, N / 16, SMEM, o, &per_sm, &sms);
    if (e != cudaSuccess) return e;
    const long long g = grid_for((a.c.m + 1) / 2, per_sm, sms, cap);
    *grid = (int)g;
    kern<<<(unsigned)g, N / 16, SMEM, s>>>(a);
    return cudaGetLastError();
}

template <int N, int DT, int INTERP>
cudaError_t bwd_variant(const AfArgs& a, cudaStream_t s, int cap, int* grid) {
    constexpr int SMEM = AfLayout<N, DT>::TOTAL;
    static Occ o;
    int per_sm = 0, sms = 0;
    auto kern = af_backward_kernel<N, DT, INTERP>;
    cudaError_t e = occupancy(kern, N / 16, SMEM, o, &per_sm, &sms);
    if (e != cudaSuccess) return e;
    const long long g = grid_for((a.c.m + 1) / 2, per_sm, sms, cap);
    *grid = (int)g;
    kern<<<(unsigned)g, N / 16, SMEM, s>>>(a);
    return cudaGetLastError();
}

template <int N, int DT>
cudaError_t dispatch(bool backward, int interp, const AfArgs& a, cudaStream_t s, int cap, int* grid) {
    switch (interp) {
        case INTERP_LINEAR:
            return backward ? bwd_variant<N, DT, INTERP_LINEAR>(a, s, cap, grid)
                            : fwd_variant<N, DT, INTERP_LINEAR>(a, s, cap, grid);
        case INTERP_CUBIC:
            return backward ? bwd_variant<N, DT, INTERP_CUBIC>(a, s, cap, grid)
                            : fwd_variant<N, DT, INTERP_CUBIC>(a, s, cap, grid);
        case INTERP_LANCZOS:
            return backward ? bwd_variant<N, DT, INTERP_LANCZOS>(a, s, cap, grid)
                            : fwd_variant<N, DT, INTERP_LANCZOS>(a, s, cap, grid);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

#define OPE_AF_CAT2(a, b) a##b
#define OPE_AF_CAT(a, b) OPE_AF_CAT2(a, b)

cudaError_t OPE_AF_CAT(af_launch_n, OPE_AF_N)(bool backward, int in_kind, int interp, const AfArgs& a,
                                              cudaStream_t s, int cap, int* grid) {
    constexpr int N = OPE_AF_N;
    switch (in_kind) {
        case IN_U8: return dispatch<N, IN_U8>(backward, interp, a, s, cap, grid);
        case IN_U16: return dispatch<N, IN_U16>(backward, interp, a, s, cap, grid);
        case IN_F32: return dispatch<N, IN_F32>(backward, interp, a, s, cap, grid);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ope_b200
