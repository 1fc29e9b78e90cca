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
