// Fixed-pattern-noise (FPN) determination and profile state of one context.
//
// Reference: CpuBackend::Impl::computeFixedPatternNoiseIfRequested
// (cpu_backend.cpp:305-357) and getMinimumVarianceMean (cpu_kernels.tpp:402-458).
// Determination here recomputes the chain over the needed A-scans in a
// statistics kernel (no complex intermediates are stored), reduces the
// per-CTA sums in a fixed order, and selects the minimum-variance segment mean
// per bin on the device, so the frame that completes a determination is
// corrected with the new profile without a host round trip.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/ope_b200.h"
#include "chain_kernel.cuh"

namespace ope_b200 {

constexpr int FPN_SEGMENTS = 8;  // cpu_backend.cpp:306

struct FpnState {
    int n = 0;
    bool requested = false;   // requestFixedPatternNoiseDetermination pending
    bool active = false;      // a determination is accumulating rows
    bool valid = false;       // d_profile holds a profile
    long long acc_rows = 0;   // rows accumulated by the active determination
    double* d_acc = nullptr;  // FPN_SEGMENTS x (n/2) x 3 sums
    double* d_partial = nullptr;
    size_t partial_cap = 0;   // doubles
    float2* d_profile = nullptr;
    std::vector<float> host_profile;
    bool host_dirty = false;
};

cudaError_t fpn_init(FpnState& st, int n);
void fpn_free(FpnState& st);
// Runs the determination work the current frame contributes (if any).
int fpn_process_frame(FpnState& st, const ope_b200_config& cfg, int in_kind, int interp, const ChainArgs& a,
                      cudaStream_t s, std::string* err);
int fpn_set_profile(FpnState& st, const float* interleaved, size_t pairs, cudaStream_t s, std::string* err);
int fpn_get_profile(FpnState& st, float* out, size_t cap_pairs, size_t* pairs, std::string* err);

cudaError_t launch_fpn_stats(int n, int in_kind, int interp, const ChainArgs& a, long long g0, long long rows,
                             long long seg_w, int gx, double* partial, cudaStream_t s);

// Enqueue the fixed-order reduction of the per-CTA partial sums into acc
// (acc += partials) and the minimum-variance selection into a profile.
cudaError_t launch_fpn_reduce(const double* partial, double* acc, int gx, int half, cudaStream_t s);
cudaError_t launch_fpn_finalize(const double* acc, float2* profile, int half, long long seg_w, cudaStream_t s);

#define OPE_B200_DECLARE_FPN_N(NN)                                                                          \
    cudaError_t launch_fpn_stats_n##NN(int in_kind, int interp, const ChainArgs& a, long long g0, long long rows, \
                                       long long seg_w, int gx, double* partial, cudaStream_t s);
OPE_B200_DECLARE_FPN_N(512)
OPE_B200_DECLARE_FPN_N(1024)
OPE_B200_DECLARE_FPN_N(2048)
OPE_B200_DECLARE_FPN_N(4096)
OPE_B200_DECLARE_FPN_N(8192)
#undef OPE_B200_DECLARE_FPN_N

}  // namespace ope_b200
