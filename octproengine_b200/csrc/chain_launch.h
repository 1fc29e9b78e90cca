// Host-side launch interface of the fused chain kernels (one translation unit
// per FFT length instantiates all input-type x interpolation variants).
#pragma once

#include <cuda_runtime.h>

#include "chain_kernel.cuh"

namespace ope_b200 {

struct LaunchInfo {
    int grid = 0;
    int block = 0;
    int smem = 0;
    int blocks_per_sm = 0;
};

// Enqueues one chain launch over a.m A-scans. `max_ctas` > 0 caps the grid.
cudaError_t launch_chain(int n, int in_kind, int interp, const ChainArgs& a, cudaStream_t stream, int max_ctas,
                         LaunchInfo* info);

#define OPE_B200_DECLARE_N(NN)                                                                                   \
    cudaError_t launch_chain_n##NN(int in_kind, int interp, const ChainArgs& a, cudaStream_t stream, int max_ctas, \
                                   LaunchInfo* info);
OPE_B200_DECLARE_N(512)
OPE_B200_DECLARE_N(1024)
OPE_B200_DECLARE_N(2048)
OPE_B200_DECLARE_N(4096)
OPE_B200_DECLARE_N(8192)
#undef OPE_B200_DECLARE_N

bool chain_length_supported(int n);

}  // namespace ope_b200
