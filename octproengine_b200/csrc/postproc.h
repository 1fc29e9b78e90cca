// Post-process background kernels (postproc.cu).
#pragma once

#include <cuda_runtime.h>

namespace ope_b200 {

// Mean output A-scan of a frame of m A-scans of s bins (float, A-scan order).
cudaError_t bg_record(const float* out, long long m, int s, float* profile, cudaStream_t st);
// Per-bin value subtracted by the chain epilogue: weight * profile + offset.
cudaError_t bg_values(const float* profile, int s, float weight, float offset, float* bgv, cudaStream_t st);
// out -= bgv per bin, for the frame that recorded the profile.
cudaError_t bg_subtract(float* out, long long m, int s, const float* bgv, cudaStream_t st);

}  // namespace ope_b200
