/*
 * FFTW3-API shim: a project-written 1-D complex DFT behind the FFTW3 calls the
 * reference CPU backend makes. Test infrastructure only (see fftw3.h).
 *
 * Algorithm: textbook iterative radix-2 decimation-in-time Cooley-Tukey for
 * power-of-two lengths (bit-reversal permutation, then log2(n) butterfly
 * stages with a precomputed twiddle table exp(s*2*pi*i*k/n), k < n/2, each
 * entry evaluated directly in double); a direct O(n^2) double-precision DFT
 * for every other length.
 */
#include "fftw3.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

struct ope_fftw_shim_plan_s {
    int n;
    int sign;
    int is_double; /* 1: plan created through the fftw_* (double) API */
    int pow2;
    void* in;
    void* out;
    int* bitrev;       /* n entries (pow2 only) */
    double* tw_d;      /* n/2 complex twiddles, interleaved (pow2) or n (generic) */
    float* tw_f;       /* same table rounded to float (pow2 only) */
    double* work_d;    /* 2n doubles */
    float* work_f;     /* 2n floats */
};

static volatile int g_precision_mode = -1; /* -1: read env on first use */

static int shim_mode(void) {
    if (g_precision_mode < 0) {
        const char* e = getenv("OPE_FFTW_SHIM_PRECISION");
        g_precision_mode = (e && strcmp(e, "f32") == 0) ? 1 : 0;
    }
    return g_precision_mode;
}

void ope_fftw_shim_set_precision(int mode) { g_precision_mode = mode ? 1 : 0; }
int ope_fftw_shim_get_precision(void) { return shim_mode(); }

static void* aligned_alloc64(size_t bytes) {
    void* p = NULL;
    if (bytes == 0) bytes = 64;
    if (posix_memalign(&p, 64, bytes) != 0) return NULL;
    return p;
}

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static struct ope_fftw_shim_plan_s* make_plan(int n, void* in, void* out, int sign, int is_double) {
    if (n <= 0) return NULL;
    struct ope_fftw_shim_plan_s* p = (struct ope_fftw_shim_plan_s*)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->n = n;
    p->sign = (sign < 0) ? -1 : 1;
    p->is_double = is_double;
    p->pow2 = is_pow2(n);
    p->in = in;
    p->out = out;
    const double two_pi = 6.283185307179586476925286766559;
    if (p->pow2) {
        int logn = 0;
        while ((1 << logn) < n) ++logn;
        p->bitrev = (int*)malloc(sizeof(int) * (size_t)n);
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int b = 0; b < logn; ++b) r |= ((i >> b) & 1) << (logn - 1 - b);
            p->bitrev[i] = r;
        }
        int half = n / 2 > 0 ? n / 2 : 1;
        p->tw_d = (double*)malloc(sizeof(double) * 2 * (size_t)half);
        p->tw_f = (float*)malloc(sizeof(float) * 2 * (size_t)half);
        for (int k = 0; k < half; ++k) {
            double a = two_pi * (double)k / (double)n;
            p->tw_d[2 * k] = cos(a);
            p->tw_d[2 * k + 1] = p->sign * sin(a);
            p->tw_f[2 * k] = (float)p->tw_d[2 * k];
            p->tw_f[2 * k + 1] = (float)p->tw_d[2 * k + 1];
        }
    } else {
        p->tw_d = (double*)malloc(sizeof(double) * 2 * (size_t)n);
        for (int k = 0; k < n; ++k) {
            double a = two_pi * (double)k / (double)n;
            p->tw_d[2 * k] = cos(a);
            p->tw_d[2 * k + 1] = p->sign * sin(a);
        }
    }
    p->work_d = (double*)aligned_alloc64(sizeof(double) * 2 * (size_t)n);
    p->work_f = (float*)aligned_alloc64(sizeof(float) * 2 * (size_t)n);
    return p;
}

/* In-place radix-2 DIT butterflies over a bit-reversed sequence (double). */
static void radix2_d(double* x, int n, const double* tw) {
    for (int h = 1; h < n; h <<= 1) {
        int step = n / (2 * h);
        for (int base = 0; base < n; base += 2 * h) {
            for (int j = 0; j < h; ++j) {
                double wr = tw[2 * j * step], wi = tw[2 * j * step + 1];
                double* a = x + 2 * (base + j);
                double* b = x + 2 * (base + j + h);
                double tr = b[0] * wr - b[1] * wi;
                double ti = b[0] * wi + b[1] * wr;
                b[0] = a[0] - tr;
                b[1] = a[1] - ti;
                a[0] += tr;
                a[1] += ti;
            }
        }
    }
}

/* Same transform evaluated entirely in float. */
static void radix2_f(float* x, int n, const float* tw) {
    for (int h = 1; h < n; h <<= 1) {
        int step = n / (2 * h);
        for (int base = 0; base < n; base += 2 * h) {
            for (int j = 0; j < h; ++j) {
                float wr = tw[2 * j * step], wi = tw[2 * j * step + 1];
                float* a = x + 2 * (base + j);
                float* b = x + 2 * (base + j + h);
                float tr = b[0] * wr - b[1] * wi;
                float ti = b[0] * wi + b[1] * wr;
                b[0] = a[0] - tr;
                b[1] = a[1] - ti;
                a[0] += tr;
                a[1] += ti;
            }
        }
    }
}

static void dft_direct_d(const double* in, double* out, int n, const double* tw) {
    for (int k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        long long idx = 0;
        for (int j = 0; j < n; ++j) {
            double wr = tw[2 * idx], wi = tw[2 * idx + 1];
            sr += in[2 * j] * wr - in[2 * j + 1] * wi;
            si += in[2 * j] * wi + in[2 * j + 1] * wr;
            idx += k;
            if (idx >= n) idx -= n;
        }
        out[2 * k] = sr;
        out[2 * k + 1] = si;
    }
}

static void execute_plan(struct ope_fftw_shim_plan_s* p) {
    const int n = p->n;
    if (p->is_double) {
        const double* in = (const double*)p->in;
        double* out = (double*)p->out;
        double* w = p->work_d;
        if (p->pow2) {
            for (int i = 0; i < n; ++i) {
                w[2 * p->bitrev[i]] = in[2 * i];
                w[2 * p->bitrev[i] + 1] = in[2 * i + 1];
            }
            radix2_d(w, n, p->tw_d);
        } else {
            dft_direct_d(in, w, n, p->tw_d);
        }
        memcpy(out, w, sizeof(double) * 2 * (size_t)n);
        return;
    }
    const float* in = (const float*)p->in;
    float* out = (float*)p->out;
    if (p->pow2 && shim_mode() == 1) {
        float* w = p->work_f;
        for (int i = 0; i < n; ++i) {
            w[2 * p->bitrev[i]] = in[2 * i];
            w[2 * p->bitrev[i] + 1] = in[2 * i + 1];
        }
        radix2_f(w, n, p->tw_f);
        memcpy(out, w, sizeof(float) * 2 * (size_t)n);
        return;
    }
    double* w = p->work_d;
    if (p->pow2) {
        for (int i = 0; i < n; ++i) {
            w[2 * p->bitrev[i]] = (double)in[2 * i];
            w[2 * p->bitrev[i] + 1] = (double)in[2 * i + 1];
        }
        radix2_d(w, n, p->tw_d);
    } else {
        double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)n);
        for (int i = 0; i < 2 * n; ++i) tmp[i] = (double)in[i];
        dft_direct_d(tmp, w, n, p->tw_d);
        free(tmp);
    }
    for (int i = 0; i < 2 * n; ++i) out[i] = (float)w[i];
}

static void destroy_plan(struct ope_fftw_shim_plan_s* p) {
    if (!p) return;
    free(p->bitrev);
    free(p->tw_d);
    free(p->tw_f);
    free(p->work_d);
    free(p->work_f);
    free(p);
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags) {
    (void)flags;
    return make_plan(n, in, out, sign, 0);
}
void fftwf_execute(const fftwf_plan p) { execute_plan(p); }
void fftwf_destroy_plan(fftwf_plan p) { destroy_plan(p); }
fftwf_complex* fftwf_alloc_complex(size_t n) { return (fftwf_complex*)aligned_alloc64(sizeof(fftwf_complex) * n); }
void fftwf_free(void* p) { free(p); }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
    (void)flags;
    return make_plan(n, in, out, sign, 1);
}
void fftw_execute(const fftw_plan p) { execute_plan(p); }
void fftw_destroy_plan(fftw_plan p) { destroy_plan(p); }
fftw_complex* fftw_alloc_complex(size_t n) { return (fftw_complex*)aligned_alloc64(sizeof(fftw_complex) * n); }
void fftw_free(void* p) { free(p); }
