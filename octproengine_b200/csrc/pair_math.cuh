// Packed two-A-scan arithmetic for the B200 chain kernels.
//
// Every thread carries the same spectral position of TWO A-scans at once: a
// value of type `cp` holds (re_a, re_b) and (im_a, im_b) as float2 pairs, and
// every operation maps onto one Blackwell packed-FP32 instruction
// (add/sub/mul/fma .rn .f32x2). Twiddles, window and phase values are shared
// by the two A-scans, so each table load serves both.
//
// All functions are __host__ __device__: the host build (used only by the CPU
// emulation test harness) evaluates the same operations with IEEE float and
// std::fma, so a host emulation of a kernel reproduces its rounding exactly.
// No operation here may be contracted or reassociated: the device side uses
// explicit .rn intrinsics, the host side must be compiled with
// -ffp-contract=off.
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#define OPE_HD __host__ __device__ __forceinline__
#else
// host-only build (CPU emulation, table builders): CUDA's vector types
#include <vector_functions.h>
#include <vector_types.h>
#define OPE_HD inline
#endif

namespace ope_b200 {

// ---------------------------------------------------------------- scalars --
OPE_HD float fmul_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
OPE_HD float fadd_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
OPE_HD float fsub_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
OPE_HD float ffma_rn(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

// ------------------------------------------------------------------ pairs --
OPE_HD float2 dup2(float v) { return make_float2(v, v); }

#if defined(__CUDA_ARCH__)
// Packed ops are issued as inline PTX with an explicit .rn modifier: PTX
// forbids contracting such mul/add into fma, which keeps the evaluation order
// (and so the rounding) exactly as written. The __f*2_rn builtins do not
// carry that guarantee in CUDA 12.9 (measured: a mul feeding an add was fused).
__device__ __forceinline__ unsigned long long f2u(float2 v) { return *reinterpret_cast<unsigned long long*>(&v); }
__device__ __forceinline__ float2 u2f(unsigned long long v) { return *reinterpret_cast<float2*>(&v); }
#endif

OPE_HD float2 add2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)));
    return u2f(d);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}

OPE_HD float2 sub2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)));
    return u2f(d);
#else
    return make_float2(a.x - b.x, a.y - b.y);
#endif
}

OPE_HD float2 mul2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)));
    return u2f(d);
#else
    return make_float2(a.x * b.x, a.y * b.y);
#endif
}

OPE_HD float2 fma2(float2 a, float2 b, float2 c) {
#if defined(__CUDA_ARCH__)
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)), "l"(f2u(c)));
    return u2f(d);
#else
    return make_float2(std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y));
#endif
}

OPE_HD float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// ------------------------------------------------------- complex pairs --
struct cp {
    float2 re;
    float2 im;
};

OPE_HD cp cpmake(float2 re, float2 im) {
    cp r;
    r.re = re;
    r.im = im;
    return r;
}
OPE_HD cp cadd(cp a, cp b) { return cpmake(add2(a.re, b.re), add2(a.im, b.im)); }
OPE_HD cp csub(cp a, cp b) { return cpmake(sub2(a.re, b.re), sub2(a.im, b.im)); }
// a + i*b
OPE_HD cp cadd_i(cp a, cp b) { return cpmake(sub2(a.re, b.im), add2(a.im, b.re)); }
// a - i*b
OPE_HD cp csub_i(cp a, cp b) { return cpmake(add2(a.re, b.im), sub2(a.im, b.re)); }
// multiply by i
OPE_HD cp cmul_i(cp a) { return cpmake(neg2(a.im), a.re); }

// a * (c + i s) with a scalar twiddle shared by both A-scans.
OPE_HD cp cmul_tw(cp a, float c, float s) {
    const float2 C = dup2(c), S = dup2(s);
    float2 re = fma2(a.re, C, mul2(a.im, dup2(-s)));
    float2 im = fma2(a.re, S, mul2(a.im, C));
    return cpmake(re, im);
}

// Exactly rounded product a*b that the compiler cannot fuse into a later add:
// fma(a, b, nz) with nz = (-0, -0) supplied at run time (a kernel argument).
// ptxas contracts a packed multiply into a following packed add even when
// both carry .rn, and folds an fma with a literal -0 back into a multiply, so
// the zero must be opaque to it. IEEE: fma(a, b, -0) == round(a*b) for all a, b.
OPE_HD float2 mul2x(float2 a, float2 b, float2 nz) { return fma2(a, b, nz); }

// ------------------------------------------- small inverse DFTs (W = e^{+2 pi i/R})
// Outputs in natural order. `NOUT` < R computes only outputs q < NOUT
// (used by the last pass, where only bins [0, N/2) are kept). Every product by
// a twiddle constant is issued as an fma into the sum it feeds, so no bare
// multiply ever reaches an add and the rounding is fixed by the source.

template <int NOUT = 2>
OPE_HD void dft2(cp* v) {
    cp a = v[0], b = v[1];
    v[0] = cadd(a, b);
    if (NOUT > 1) v[1] = csub(a, b);
}

template <int NOUT = 4>
OPE_HD void dft4(cp& a0, cp& a1, cp& a2, cp& a3) {
    cp t0 = cadd(a0, a2), t1 = csub(a0, a2);
    cp t2 = cadd(a1, a3), t3 = csub(a1, a3);
    a0 = cadd(t0, t2);
    a1 = cadd_i(t1, t3);
    if (NOUT > 2) {
        a2 = csub(t0, t2);
        a3 = csub_i(t1, t3);
    }
}

template <int NOUT = 4>
OPE_HD void dft4v(cp* v) { dft4<NOUT>(v[0], v[1], v[2], v[3]); }

// e + W8 * o  and  e - W8 * o,  W8 = h(1 + i), h = sqrt(1/2):
// W8*o = h(o.re - o.im) + i h(o.re + o.im)
OPE_HD void bfly_w8(const cp& e, const cp& o, cp& plus, cp& minus) {
    const float2 H = dup2(0.70710678118654752440f), NH = dup2(-0.70710678118654752440f);
    const float2 s = sub2(o.re, o.im), u = add2(o.re, o.im);
    plus = cpmake(fma2(s, H, e.re), fma2(u, H, e.im));
    minus = cpmake(fma2(s, NH, e.re), fma2(u, NH, e.im));
}
// e + W8^3 * o  and  e - W8^3 * o,  W8^3 = h(-1 + i):
// W8^3*o = -h(o.re + o.im) + i h(o.re - o.im)
OPE_HD void bfly_w83(const cp& e, const cp& o, cp& plus, cp& minus) {
    const float2 H = dup2(0.70710678118654752440f), NH = dup2(-0.70710678118654752440f);
    const float2 s = sub2(o.re, o.im), u = add2(o.re, o.im);
    plus = cpmake(fma2(u, NH, e.re), fma2(s, H, e.im));
    minus = cpmake(fma2(u, H, e.re), fma2(s, NH, e.im));
}

template <int NOUT = 8>
OPE_HD void dft8(cp* v) {
    // radix-2 split: E = DFT4(even), O = DFT4(odd); X_q = E_q + W8^q O_q
    cp e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    cp o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<4>(e0, e1, e2, e3);
    dft4<4>(o0, o1, o2, o3);
    cp p1, m1, p3, m3;
    bfly_w8(e1, o1, p1, m1);
    bfly_w83(e3, o3, p3, m3);
    v[0] = cadd(e0, o0);
    v[1] = p1;
    v[2] = cadd_i(e2, o2);
    v[3] = p3;
    if (NOUT > 4) {
        v[4] = csub(e0, o0);
        v[5] = m1;
        v[6] = csub_i(e2, o2);
        v[7] = m3;
    }
}

template <int NOUT = 16>
OPE_HD void dft16(cp* v) {
    // 4x4 decomposition: n = 4*n1 + n2, k = k1 + 4*k2.
    // Stage 1: F[n2] = DFT4 over n1. Stage 2, per k1: DFT4 over n2 of
    // W16^(n2*k1) F[n2][k1]. General twiddles (W^1, W^3, W^9) are fma-based
    // complex products; W^2 and W^6 (multiples of h(1 +- i)) are folded into
    // the first butterfly of the stage-2 DFT4 as fmas; W^4 = i is a swap.
    const float C1 = 0.92387953251128675613f;  // cos(pi/8)
    const float S1 = 0.38268343236508977173f;  // sin(pi/8)
    cp f[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        f[n2][0] = v[n2];
        f[n2][1] = v[4 + n2];
        f[n2][2] = v[8 + n2];
        f[n2][3] = v[12 + n2];
        dft4<4>(f[n2][0], f[n2][1], f[n2][2], f[n2][3]);
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        cp a0 = f[0][k1], a1 = f[1][k1], a2 = f[2][k1], a3 = f[3][k1];
        cp t0, t1, t2, t3;
        if (k1 == 0) {
            t0 = cadd(a0, a2);
            t1 = csub(a0, a2);
            t2 = cadd(a1, a3);
            t3 = csub(a1, a3);
        } else if (k1 == 1) {
            a1 = cmul_tw(a1, C1, S1);  // W^1
            a3 = cmul_tw(a3, S1, C1);  // W^3
            bfly_w8(a0, a2, t0, t1);   // a0 +- W^2 a2
            t2 = cadd(a1, a3);
            t3 = csub(a1, a3);
        } else if (k1 == 2) {
            // a1*W^2, a2*W^4 = i a2, a3*W^6: t2 = W^2 (a1 + i a3), t3 = W^2 (a1 - i a3)
            t0 = cadd_i(a0, a2);
            t1 = csub_i(a0, a2);
            const cp b = cadd_i(a1, a3), c = csub_i(a1, a3);
            // stage-2 outputs: X0 = t0 + W^2 b, X2 = t0 - W^2 b, X1 = t1 + i W^2 c, X3 = t1 - i W^2 c;
            // i W^2 = W^6
            cp x0, x2, x1, x3;
            bfly_w8(t0, b, x0, x2);
            bfly_w83(t1, c, x1, x3);
            v[2] = x0;
            v[6] = x1;
            if (NOUT > 8) {
                v[10] = x2;
                v[14] = x3;
            }
            continue;
        } else {
            a1 = cmul_tw(a1, S1, C1);     // W^3
            a3 = cmul_tw(a3, -C1, -S1);   // W^9
            bfly_w83(a0, a2, t0, t1);     // a0 +- W^6 a2
            t2 = cadd(a1, a3);
            t3 = csub(a1, a3);
        }
        v[k1] = cadd(t0, t2);
        v[k1 + 4] = cadd_i(t1, t3);
        if (NOUT > 8) {
            v[k1 + 8] = csub(t0, t2);
            v[k1 + 12] = csub_i(t1, t3);
        }
    }
}

}  // namespace ope_b200
