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

OPE_HD float2 add2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}

OPE_HD float2 sub2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    unsigned long long ra = *reinterpret_cast<unsigned long long*>(&a);
    unsigned long long rb = *reinterpret_cast<unsigned long long*>(&b);
    unsigned long long rd;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
    return *reinterpret_cast<float2*>(&rd);
#else
    return make_float2(a.x - b.x, a.y - b.y);
#endif
}

OPE_HD float2 mul2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    return __fmul2_rn(a, b);
#else
    return make_float2(a.x * b.x, a.y * b.y);
#endif
}

OPE_HD float2 fma2(float2 a, float2 b, float2 c) {
#if defined(__CUDA_ARCH__)
    return __ffma2_rn(a, b, c);
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

// a * (h + i h) and a * (-h + i h), h = sqrt(1/2)
OPE_HD cp cmul_w8(cp a) {
    const float2 H = dup2(0.70710678118654752440f);
    return cpmake(mul2(sub2(a.re, a.im), H), mul2(add2(a.re, a.im), H));
}
OPE_HD cp cmul_w8_3(cp a) {
    const float2 H = dup2(0.70710678118654752440f);
    return cpmake(mul2(neg2(add2(a.re, a.im)), H), mul2(sub2(a.re, a.im), H));
}

// ------------------------------------------- small inverse DFTs (W = e^{+2 pi i/R})
// Outputs in natural order. `NOUT` < R computes only outputs q < NOUT
// (used by the last pass, where only bins [0, N/2) are kept).

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

template <int NOUT = 8>
OPE_HD void dft8(cp* v) {
    // radix-2 split: E = DFT4(even), O = DFT4(odd); X_q = E_q + W8^q O_q
    cp e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    cp o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<4>(e0, e1, e2, e3);
    dft4<4>(o0, o1, o2, o3);
    o1 = cmul_w8(o1);
    o2 = cmul_i(o2);
    o3 = cmul_w8_3(o3);
    v[0] = cadd(e0, o0);
    v[1] = cadd(e1, o1);
    v[2] = cadd(e2, o2);
    v[3] = cadd(e3, o3);
    if (NOUT > 4) {
        v[4] = csub(e0, o0);
        v[5] = csub(e1, o1);
        v[6] = csub(e2, o2);
        v[7] = csub(e3, o3);
    }
}

template <int NOUT = 16>
OPE_HD void dft16(cp* v) {
    // 4x4 decomposition: n = 4*n1 + n2, k = k1 + 4*k2
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
    // twiddles W16^(n2*k1)
    f[1][1] = cmul_tw(f[1][1], C1, S1);     // W^1
    f[1][2] = cmul_w8(f[1][2]);             // W^2
    f[1][3] = cmul_tw(f[1][3], S1, C1);     // W^3
    f[2][1] = cmul_w8(f[2][1]);             // W^2
    f[2][2] = cmul_i(f[2][2]);              // W^4
    f[2][3] = cmul_w8_3(f[2][3]);           // W^6
    f[3][1] = cmul_tw(f[3][1], S1, C1);     // W^3
    f[3][2] = cmul_w8_3(f[3][2]);           // W^6
    f[3][3] = cmul_tw(f[3][3], -C1, -S1);   // W^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        cp a0 = f[0][k1], a1 = f[1][k1], a2 = f[2][k1], a3 = f[3][k1];
        if (NOUT > 8) {
            dft4<4>(a0, a1, a2, a3);
            v[k1] = a0;
            v[k1 + 4] = a1;
            v[k1 + 8] = a2;
            v[k1 + 12] = a3;
        } else {
            dft4<2>(a0, a1, a2, a3);
            v[k1] = a0;
            v[k1 + 4] = a1;
        }
    }
}

}  // namespace ope_b200
