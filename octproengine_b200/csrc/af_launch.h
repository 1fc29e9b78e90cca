// Host-side launch interface of the autofocus kernels (one translation unit
// per FFT length).
#pragma once

#include <cuda_runtime.h>

namespace ope_b200 {

struct AfArgs;

// Enqueues the forward (backward = false) or adjoint kernel over a.c.m
// A-scans with at most `cap` CTAs; *grid receives the CTA count (one partial
// record per CTA).
#define OPE_AF_DECLARE_N(NN)                                                                              \
    cudaError_t af_launch_n##NN(bool backward, int in_kind, int interp, const AfArgs& a, cudaStream_t s, \
                                int cap, int* grid);
OPE_AF_DECLARE_N(1024)
OPE_AF_DECLARE_N(2048)
OPE_AF_DECLARE_N(4096)
#undef OPE_AF_DECLARE_N

}  // namespace ope_b200
