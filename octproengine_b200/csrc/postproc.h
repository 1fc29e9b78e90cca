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
// Sinusoidal scan correction curve of `length` A-scans per B-scan (device acosf).
cudaError_t sin_curve(float* curve, int length, cudaStream_t st);
// out = sinusoidal correction of `in` (m A-scans of `width` bins, `height`
// A-scans per B-scan), then minus bgv per bin when bgv is set.
cudaError_t sin_correct(float* out, const float* in, const float* curve, int width, int height, long long m,
                        const float* bgv, cudaStream_t st);

}  // namespace ope_b200
