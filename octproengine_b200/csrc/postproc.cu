// Post-process background of the chain output (PostProcessingParameters::
// backgroundRemoval): recording the mean output A-scan of a frame and the
// per-bin value the chain epilogue subtracts. Restates
// CpuBackend::Impl::recordPostProcessBackground (cpu_backend.cpp:105-118) and
// applyPostProcessBackgroundSubtraction (cpu_kernels.tpp:381-400) with the
// same float operations in the same order.
#include <cuda_runtime.h>

#include "postproc.h"

namespace ope_b200 {

// profile[i] = (sum over A-scans a = 0..m-1, in order, of out[a*s + i]) / m,
// accumulated in float like the reference: one thread per bin, the loads of
// successive A-scans are independent and kept in flight.
__global__ void bg_record_kernel(const float* __restrict__ out, long long m, int s, float* __restrict__ profile) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s) return;
    float sum = 0.0f;
    const float* p = out + i;
#pragma unroll 8
    for (long long a = 0; a < m; ++a) sum = __fadd_rn(sum, __ldg(p + a * s));
    profile[i] = __fdiv_rn(sum, static_cast<float>(m));
}

// bgv[i] = weight * profile[i] + offset, rounded after each operation.
__global__ void bg_value_kernel(const float* __restrict__ profile, int s, float weight, float offset,
                                float* __restrict__ bgv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < s) bgv[i] = __fadd_rn(__fmul_rn(weight, profile[i]), offset);
}

// out[a*s + i] -= bgv[i] for the frame that recorded the profile.
__global__ void bg_subtract_kernel(float* __restrict__ out, long long total, int s, const float* __restrict__ bgv) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x)
        out[k] = __fsub_rn(out[k], __ldg(bgv + (k % s)));
}

cudaError_t bg_record(const float* out, long long m, int s, float* profile, cudaStream_t st) {
    bg_record_kernel<<<(s + 127) / 128, 128, 0, st>>>(out, m, s, profile);
    return cudaGetLastError();
}

cudaError_t bg_values(const float* profile, int s, float weight, float offset, float* bgv, cudaStream_t st) {
    bg_value_kernel<<<(s + 255) / 256, 256, 0, st>>>(profile, s, weight, offset, bgv);
    return cudaGetLastError();
}

cudaError_t bg_subtract(float* out, long long m, int s, const float* bgv, cudaStream_t st) {
    const long long total = m * s;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    bg_subtract_kernel<<<(unsigned)blocks, 256, 0, st>>>(out, total, s, bgv);
    return cudaGetLastError();
}

}  // namespace ope_b200

namespace ope_b200 {

// fillSinusoidalScanCorrectionCurve (cuda_kernels.cu:433-438), the same
// mixed float/double expression: curve[k] = (L/pi) acos(1 - 2k/L), L = A-scans
// per B-scan, with the device acosf.
__global__ void sin_curve_kernel(float* curve, int length) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= length) return;
    const double arg = 1.0 - ((2.0 * (double)(float)k) / (double)(float)length);
    curve[k] = (float)(((double)(float)length / 3.14159265358979323846) * (double)acosf((float)arg));
}

// sinusoidalScanCorrection (cuda_kernels.cu:408-431): output A-scan k of a
// B-scan interpolates linearly between input A-scans (int)x and (int)x + 1,
// x = curve[k], bin by bin; the last A-scan of the buffer keeps its value.
// The interpolation is fused into one fma as a default CUDA build does.
// With bgv set, the post-process background is subtracted afterwards
// (the reference runs it as the next step, cuda_backend.cu:696-743).
__global__ void sin_correct_kernel(float* __restrict__ out, const float* __restrict__ in,
                                   const float* __restrict__ curve, int width, int height, long long samples,
                                   const float* __restrict__ bgv) {
    for (long long index = blockIdx.x * (long long)blockDim.x + threadIdx.x; index < samples;
         index += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(index % width);
        float v;
        if (index < samples - width) {
            const int k = (int)((index / width) % height);
            const long long l = index / ((long long)width * height);
            const float x = __ldg(curve + k);
            const long long x0 = (long long)(int)x * width + j + l * width * height;
            const float f0 = __ldg(in + x0), f1 = __ldg(in + x0 + width);
            v = __fmaf_rn(__fsub_rn(f1, f0), __fsub_rn(x, (float)(int)x), f0);
        } else {
            v = __ldg(in + index);
        }
        if (bgv) v = __fsub_rn(v, __ldg(bgv + j));
        out[index] = v;
    }
}

cudaError_t sin_curve(float* curve, int length, cudaStream_t st) {
    sin_curve_kernel<<<(length + 127) / 128, 128, 0, st>>>(curve, length);
    return cudaGetLastError();
}

cudaError_t sin_correct(float* out, const float* in, const float* curve, int width, int height, long long m,
                        const float* bgv, cudaStream_t st) {
    const long long samples = m * width;
    long long blocks = (samples + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    sin_correct_kernel<<<(unsigned)blocks, 256, 0, st>>>(out, in, curve, width, height, samples, bgv);
    return cudaGetLastError();
}

}  // namespace ope_b200
