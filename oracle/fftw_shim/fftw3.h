/*
 * Minimal FFTW3-API shim used ONLY to compile the reference CPU backend as a
 * test oracle (FFTW3 itself is not installed on the build machines).
 *
 * This is test infrastructure, not product code. It declares exactly the part
 * of the FFTW3 single/double precision API that the reference CPU backend
 * touches (src/backends/cpu/cpu_backend.cpp:377-391,93-101 and
 * src/backends/cpu/cpu_kernels.tpp:246-259,278-291): plan creation for a 1-D
 * complex DFT, execution, plan destruction and aligned complex allocation.
 *
 * The transform is the one FFTW defines: for sign s (FFTW_FORWARD = -1,
 * FFTW_BACKWARD = +1) and length n,  out[k] = sum_j in[j] * exp(s*2*pi*i*j*k/n),
 * unnormalised. Precision of the single-precision path is selectable (see
 * fftw_shim.c): "f64" (default) evaluates in double and rounds once to float,
 * "f32" evaluates an iterative radix-2 transform in float like a typical FP32
 * library FFT would. Every report that uses this shim must say
 * "FFT = project shim, not FFTW".
 */
#ifndef OPE_FFTW_SHIM_FFTW3_H
#define OPE_FFTW_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef float fftwf_complex[2];
typedef double fftw_complex[2];

typedef struct ope_fftw_shim_plan_s* fftwf_plan;
typedef struct ope_fftw_shim_plan_s* fftw_plan;

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
fftwf_complex* fftwf_alloc_complex(size_t n);
void fftwf_free(void* p);

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);

/* Shim-only controls: 0 = evaluate single-precision plans in double (default),
 * 1 = evaluate them in float (radix-2, FP32 arithmetic). */
void ope_fftw_shim_set_precision(int mode);
int ope_fftw_shim_get_precision(void);

#ifdef __cplusplus
}
#endif

#endif
