// Host-side builders of the device tables the chain kernels read. Pure C++
// (no CUDA runtime calls) so the same code serves the C ABI and the CPU
// emulation harness of the tests.
#pragma once

#include <vector>

#include "chain_kernel.cuh"

namespace ope_b200 {

// lanczosKernel<float>(x, 8) of the reference (cpu_kernels.tpp:148-162),
// evaluated with the same float operations.
float lanczos8(float x);

// Twiddles of the Stockham passes of radix schedule `sched` (Sched<N, S>: the
// short pass last for 0, as pass sched - 1 otherwise),
// per pass a block of (R-1) x NS entries W_N^(r k N/(NS R)) (see
// Sched::tw_off), evaluated in double and rounded once.
std::vector<float2> build_twiddles(int n, int sched = 0);

// kLinearizationLinear indices and fractions (cpu_kernels.tpp:95-110):
// {n1 + SPEC_PAD, bits of float(nx - n1)}.
std::vector<int2> build_linear_table(const float* curve, int n);

// kLinearizationCubic indices (cpu_kernels.tpp:124-145): n0 and n1, packed
// 16-bit and offset by SPEC_PAD, and pos as float bits (the kernel reads taps
// n1+1, n1+2 and forms pos*pos).
std::vector<int2> build_cubic_table(const float* curve, int n);

// kLinearizationLanczos taps (cpu_kernels.tpp:176-195): per output index the
// first gathered index (+ SPEC_PAD) and 16 weights (tap-major, 16 x n).
void build_lanczos_table(const float* curve, int n, std::vector<int>& base, std::vector<float>& w);

// Response of the chain up to the inverse DFT to a constant spectrum of 1:
// D[k] = sum_j g_j w_j (cos_j + i sin_j) exp(+2 pi i j k / N), k < N/2,
// in float64 (g_j = 1 for no/linear/cubic resampling, the sum of the 16
// Lanczos weights of output j otherwise). Used by the exact DC split.
std::vector<float2> build_dc_response(int n, int interp, const float* lanczos_w, const float* window,
                                      const float* cos_sin);

// {w cos, w sin} per sample, products in double rounded once; a missing
// window is 1, a missing phase (cos 1, sin 0).
std::vector<float2> build_window_phase(const float* window, const float* cos_sin, int n);

// Output affine constants of logScaleAndTruncate / linearScaleAndTruncate
// (cpu_kernels.tpp:301-378) folded for the kernel epilogue.
void scaling_constants(bool log_scaling, float gmin, float gmax, float addend, float mult, int n, ChainArgs& a);

}  // namespace ope_b200
