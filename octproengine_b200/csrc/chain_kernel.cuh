// Fused per-A-scan OCT chain for B200 (sm_100a).
//
// One CTA ("team") of T = N/16 threads processes one PAIR of A-scans at a time
// in a persistent loop; the two A-scans ride in the two lanes of packed f32x2
// registers (pair_math.cuh). Per pair:
//
//   raw rows --(cp.async.bulk, double-buffered, mbarrier)--> smem
//   unpack to float pairs (+ rolling-average DC removal)       -> smem "spec"
//   k-linearisation gather (none / linear / cubic / Lanczos-8)  -> registers
//   x window x (cos, sin) of the dispersion phase              -> registers
//   inverse DFT: Stockham radix-16 passes through swizzled smem -> registers
//   FPN subtraction, |X|^2, log10 or linear scaling, affine    -> HBM (bins < N/2)
//
// Each raw spectrum is read from HBM once and each output once; everything in
// between stays on chip. The stage semantics follow the reference CPU backend
// (src/backends/cpu/cpu_kernels.tpp:24-378, cpu_backend.cpp:169-302); see the
// notes at each phase.
//
// The phase functions are __host__ __device__ and take the thread index
// explicitly, so the CPU emulation harness (tests/emu) runs this exact code
// thread by thread between emulated barriers.
#pragma once

#include <cstring>

#include "pair_math.cuh"

#if !defined(__CUDACC__)
#include <cassert>
#define OPE_SMEM_CHECK(cond) assert(cond)
#else
#define OPE_SMEM_CHECK(cond) ((void)0)
#endif

namespace ope_b200 {

// Input element types of the fused chain.
enum InputKind : int { IN_U8 = 0, IN_U16 = 1, IN_U32 = 2, IN_F32 = 3 };
// Resampling (k-linearisation) variants; the non-NONE values follow
// ope::InterpolationMethod + 1 (include/processorconfiguration.h:16-20).
enum InterpKind : int { INTERP_NONE = 0, INTERP_LINEAR = 1, INTERP_CUBIC = 2, INTERP_LANCZOS = 3 };

// Replicated-edge padding of the unpacked spectrum: gathers at indices in
// [-PAD, N+PAD) read the clamped edge value, which is how the reference clamps
// (cpu_kernels.tpp:101-102,132-135,187-188).
constexpr int SPEC_PAD = 16;

// Device status word bits.
constexpr int STATUS_MBAR_TIMEOUT = 1;  // a bounded wait for an input copy ran out
constexpr int STATUS_COPY_PENDING = 2;  // ... and the copy had still not landed after a second bound

struct ChainArgs {
    const void* in;      // m rows x n samples
    float* out;          // m rows x n/2 bins
    long long m;         // A-scans in this buffer
    const float2* tw;    // W_N^j = (cos, sin)(2 pi j / N), j < N
    const int2* lin;     // LINEAR: {n1 + PAD, float bits of (nx - n1)}
    const int2* cub;     // CUBIC: {n0 | n1<<16 (both +PAD), pos bits}; taps n2, n3 are n1+1, n1+2
    const int* lz_base;  // LANCZOS: first tap index + PAD
    const float* lz_w;   // LANCZOS: 16 x N tap weights, tap-major
    const float2* wph;   // {w*cos, w*sin} (window folded into the phase)
    const float2* fpn;   // N/2 complex fixed-pattern profile, or nullptr
    int dc_window;       // rolling-average half window W; 0 = off
    int log_mode;        // 1: logarithmic, 0: linear
    int auto_minmax;     // log mode with grayscaleMin == grayscaleMax
    float k_a, k_b;      // log: out = k_a*log2|X|^2 + k_b; linear: out = k_a*|X| + k_b
    float mult, addend;  // auto-minmax affine
    int flip;            // B-scan flip (output row remap)
    int ascans_per_bscan;
    int bscans;          // B-scans in this buffer
    int* status;         // device error word (may be nullptr)
    unsigned long long timeout_ns;
    float2* bins_out;    // if set: write complex bins [0, N/2) per A-scan instead of the image
    int debug_skip_first_copy;  // test hook: never issue the first bulk copy (exercises the timeout path)
    float neg_zero;      // -0.0f, passed at run time (see mul2x in pair_math.cuh)
    // Exact DC split: when set, each A-scan's integer mean c is subtracted
    // exactly before the chain and c * dc_resp[k] added back after the DFT.
    // dc_resp[k] (k < N/2) is the chain's response to a constant 1 spectrum,
    // evaluated in float64; the chain is linear up to the DFT, so the result
    // is the same quantity computed with a far smaller float32 error floor.
    const float2* dc_resp;
    float* resampled_out;  // test hook (CPU emulation only): k-linearised spectrum of the last pair
    // Post-process background (applyPostProcessBackgroundSubtraction,
    // cpu_kernels.tpp:381-400): when set, bgv[b] = weight * profile[b] + offset
    // is subtracted from every output value of bin b after the scaling.
    const float* bgv;
    int bitshift;  // DataParameters::bitshift for 8/16-bit samples: each sample >> 4 before the chain
    int debug_abort_first_wait;  // test hook: treat the first wait as run out although its copy was issued
    int dc_ref_order;  // rolling-average DC removal with the reference's sequential float prefix sum
};

template <int N_>
struct Plan {
    static constexpr int N = N_;
    static_assert(N >= 256 && N <= 8192 && (N & (N - 1)) == 0, "N must be a power of two in [256, 8192]");
    static constexpr int T = N / 16;  // threads per team
    static constexpr int LOG2N = (N == 256) ? 8 : (N == 512) ? 9 : (N == 1024) ? 10 : (N == 2048) ? 11 : (N == 4096) ? 12 : 13;
    static constexpr int NPASS = (LOG2N + 3) / 4;
    static constexpr int LASTR = 1 << (LOG2N - 4 * (NPASS - 1));
    static constexpr int HALF = N / 2;
    // exchange buffer: one float4 per element, slots swizzled by xslot
    static constexpr int EXCH_ELEMS = N;
};

// Exchange-buffer slot of element e: the low three bits (the 16-byte bank
// group) XORed with bits 4..6. Lanes storing elements 16 apart (the first
// radix-16 pass) land in distinct bank groups, and runs of 8 consecutive
// elements (every load, and the stores of later passes) stay conflict-free,
// with no padding slots: the same bank-group spread as one pad slot per 16
// elements on every radix schedule, in N slots instead of N + N/16.
OPE_HD int xslot(int e) { return e ^ ((e >> 4) & 7); }

OPE_HD float bits_f(int b) {
#if defined(__CUDA_ARCH__)
    return __int_as_float(b);
#else
    float f;
    std::memcpy(&f, &b, 4);
    return f;
#endif
}

template <int DT>
struct InTraits;
template <>
struct InTraits<IN_U8> { using raw_t = unsigned char; using sum_t = int; };
template <>
struct InTraits<IN_U16> { using raw_t = unsigned short; using sum_t = int; };
template <>
struct InTraits<IN_U32> { using raw_t = unsigned int; using sum_t = long long; };
template <>
struct InTraits<IN_F32> { using raw_t = float; using sum_t = float; };

// Shared-memory layout of one team (bytes).
template <int N, int DT>
struct Layout {
    using sum_t = typename InTraits<DT>::sum_t;
    using raw_t = typename InTraits<DT>::raw_t;
    static constexpr int SPEC_BYTES = (N + 2 * SPEC_PAD) * 8;        // float2 pairs
    // prefix sums, 2 rows, two pad words per 32 (pfx_idx): conflict-free writes and reads;
    // rounded to 16 bytes so that the scan scratch after it holds doubles aligned
    static constexpr int PFX_BYTES =
        (((N + 1) * 2 + 2 * (((N + 1) * 2) / 32) + 2) * (int)sizeof(sum_t) + 15) / 16 * 16;
    static constexpr int EXCH_BYTES_RAW = Plan<N>::EXCH_ELEMS * 16;
    static constexpr int WORK_BYTES = (EXCH_BYTES_RAW > SPEC_BYTES + PFX_BYTES + 256)
                                          ? EXCH_BYTES_RAW
                                          : SPEC_BYTES + PFX_BYTES + 256;
    static constexpr int STAGE_BYTES = 2 * N * (int)sizeof(raw_t);  // two raw rows
    static constexpr int OFF_SPEC = 0;
    static constexpr int OFF_PFX = SPEC_BYTES;
    static constexpr int OFF_SCAN = SPEC_BYTES + PFX_BYTES;  // 256 B of scan scratch
    static constexpr int OFF_EXCH = 0;
    static constexpr int OFF_STAGE = ((WORK_BYTES + 127) / 128) * 128;
    static constexpr int OFF_MBAR = OFF_STAGE + STAGE_BYTES;  // one stage: refilled once unpacked
    static constexpr int TOTAL = OFF_MBAR + 64;
    static_assert(OFF_PFX % 16 == 0 && OFF_SCAN % 16 == 0 && OFF_STAGE % 128 == 0 && OFF_MBAR % 16 == 0,
                  "shared-memory regions must stay aligned for their widest accesses");
};

// ------------------------------------------------------------------ unpack --

OPE_HD float u16_to_float(unsigned v) { return (float)v; }

// Eight consecutive samples of both rows of a pair -> float pairs.
template <int DT>
OPE_HD void load_chunk8(const unsigned char* stage, int n, int c, float2* vals) {
    using raw_t = typename InTraits<DT>::raw_t;
    const raw_t* ra = reinterpret_cast<const raw_t*>(stage);
    const raw_t* rb = ra + n;
#if defined(__CUDA_ARCH__)
    if (DT == IN_U16) {
        uint4 wa = *reinterpret_cast<const uint4*>(ra + 8 * c);
        uint4 wb = *reinterpret_cast<const uint4*>(rb + 8 * c);
        const unsigned wa4[4] = {wa.x, wa.y, wa.z, wa.w};
        const unsigned wb4[4] = {wb.x, wb.y, wb.z, wb.w};
        const float2 magic = dup2(8388608.0f);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            // 0x4B00_0000 | u16 is the float 2^23 + u; subtracting 2^23 is exact.
            float lo_a = __uint_as_float(__byte_perm(wa4[k], 0x4B00u, 0x5410));
            float lo_b = __uint_as_float(__byte_perm(wb4[k], 0x4B00u, 0x5410));
            float hi_a = __uint_as_float(__byte_perm(wa4[k], 0x4B00u, 0x5432));
            float hi_b = __uint_as_float(__byte_perm(wb4[k], 0x4B00u, 0x5432));
            vals[2 * k] = sub2(make_float2(lo_a, lo_b), magic);
            vals[2 * k + 1] = sub2(make_float2(hi_a, hi_b), magic);
        }
        return;
    }
    if (DT == IN_U8) {
        uint2 wa = *reinterpret_cast<const uint2*>(ra + 8 * c);
        uint2 wb = *reinterpret_cast<const uint2*>(rb + 8 * c);
        const unsigned wa2[2] = {wa.x, wa.y};
        const unsigned wb2[2] = {wb.x, wb.y};
        const float2 magic = dup2(8388608.0f);
        const unsigned sel[4] = {0x5440, 0x5441, 0x5442, 0x5443};
#pragma unroll
        for (int k = 0; k < 2; ++k)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float a = __uint_as_float(__byte_perm(wa2[k], 0x4B00u, sel[j]));
                float b = __uint_as_float(__byte_perm(wb2[k], 0x4B00u, sel[j]));
                vals[4 * k + j] = sub2(make_float2(a, b), magic);
            }
        return;
    }
#endif
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        raw_t a = ra[8 * c + i];
        raw_t b = rb[8 * c + i];
        if (DT == IN_U32) {
#if defined(__CUDA_ARCH__)
            vals[i] = make_float2(__uint2float_rn((unsigned)a), __uint2float_rn((unsigned)b));
#else
            vals[i] = make_float2((float)(unsigned)a, (float)(unsigned)b);
#endif
        } else {
            vals[i] = make_float2((float)a, (float)b);
        }
    }
}

template <int DT>
OPE_HD void load_raw_pair(const unsigned char* stage, int n, int i, typename InTraits<DT>::sum_t& sa,
                          typename InTraits<DT>::sum_t& sb) {
    using raw_t = typename InTraits<DT>::raw_t;
    using sum_t = typename InTraits<DT>::sum_t;
    const raw_t* ra = reinterpret_cast<const raw_t*>(stage);
    sa = (sum_t)ra[i];
    sb = (sum_t)ra[n + i];
}

// Samples 2p and 2p+1 of both rows: out[0] = (a[2p], b[2p]), out[1] = (a[2p+1], b[2p+1]).
template <int DT>
OPE_HD void load_pos2(const unsigned char* stage, int n, int p, float2* out) {
    using raw_t = typename InTraits<DT>::raw_t;
    const raw_t* ra = reinterpret_cast<const raw_t*>(stage);
    const raw_t* rb = ra + n;
#if defined(__CUDA_ARCH__)
    if (DT == IN_U16) {
        const unsigned wa = *reinterpret_cast<const unsigned*>(ra + 2 * p);
        const unsigned wb = *reinterpret_cast<const unsigned*>(rb + 2 * p);
        const float2 magic = dup2(8388608.0f);
        out[0] = sub2(make_float2(__uint_as_float(__byte_perm(wa, 0x4B00u, 0x5410)),
                                  __uint_as_float(__byte_perm(wb, 0x4B00u, 0x5410))), magic);
        out[1] = sub2(make_float2(__uint_as_float(__byte_perm(wa, 0x4B00u, 0x5432)),
                                  __uint_as_float(__byte_perm(wb, 0x4B00u, 0x5432))), magic);
        return;
    }
    if (DT == IN_U8) {
        const unsigned wa = *reinterpret_cast<const unsigned short*>(ra + 2 * p);
        const unsigned wb = *reinterpret_cast<const unsigned short*>(rb + 2 * p);
        const float2 magic = dup2(8388608.0f);
        out[0] = sub2(make_float2(__uint_as_float(__byte_perm(wa, 0x4B00u, 0x5440)),
                                  __uint_as_float(__byte_perm(wb, 0x4B00u, 0x5440))), magic);
        out[1] = sub2(make_float2(__uint_as_float(__byte_perm(wa, 0x4B00u, 0x5441)),
                                  __uint_as_float(__byte_perm(wb, 0x4B00u, 0x5441))), magic);
        return;
    }
#endif
    for (int i = 0; i < 2; ++i) {
        const raw_t a = ra[2 * p + i], b = rb[2 * p + i];
        if (DT == IN_U32) {
#if defined(__CUDA_ARCH__)
            out[i] = make_float2(__uint2float_rn((unsigned)a), __uint2float_rn((unsigned)b));
#else
            out[i] = make_float2((float)(unsigned)a, (float)(unsigned)b);
#endif
        } else {
            out[i] = make_float2((float)a, (float)b);
        }
    }
}

// Plain unpack (no DC removal): spec[PAD + k] = (a[k], b[k]) for k < N, with
// replicated edges. Thread t handles the sample pairs p = t + k*T (k < 8),
// i.e. samples 2p and 2p+1: consecutive lanes read consecutive 32-bit raw
// words and write consecutive 16-byte spec slots (no bank conflicts).
template <int N, int DT>
OPE_HD void phase_unpack(int t, const unsigned char* stage, float2* spec) {
    constexpr int T = Plan<N>::T;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int p = t + k * T;
        float2 v[2];
        load_pos2<DT>(stage, N, p, v);
        OPE_SMEM_CHECK(SPEC_PAD + 2 * p + 1 < N + 2 * SPEC_PAD);
        *reinterpret_cast<float4*>(&spec[SPEC_PAD + 2 * p]) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
        if (p == 0)
            for (int e = 0; e < SPEC_PAD; ++e) spec[e] = v[0];
        if (p == N / 2 - 1)
            for (int e = 0; e < SPEC_PAD; ++e) spec[SPEC_PAD + N + e] = v[1];
    }
}

// Exact DC split, step A: thread t loads its two 8-sample chunks (kept in
// registers across the team reduction) and sums each row in double.
// Sum type of the split level: exact integers for 8/16-bit samples (at most
// 8192 * 65535 < 2^31), double otherwise.
template <int DT>
struct SplitSum { using type = double; };
template <>
struct SplitSum<IN_U8> { using type = int; };
template <>
struct SplitSum<IN_U16> { using type = int; };

template <int N, int DT>
OPE_HD void phase_split_load(int t, const unsigned char* stage, float2* vals, typename SplitSum<DT>::type* sa,
                             typename SplitSum<DT>::type* sb) {
    using S = typename SplitSum<DT>::type;
    constexpr int T = Plan<N>::T;
    float fa = 0.0f, fb = 0.0f;  // exact: 16 samples below 2^16 sum below 2^24
    S a = 0, b = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        load_pos2<DT>(stage, N, t + k * T, vals + 2 * k);
        if (DT == IN_U8 || DT == IN_U16) {
            fa = fadd_rn(fadd_rn(fa, vals[2 * k].x), vals[2 * k + 1].x);
            fb = fadd_rn(fadd_rn(fb, vals[2 * k].y), vals[2 * k + 1].y);
        } else {
            a += (S)vals[2 * k].x;
            b += (S)vals[2 * k].y;
            a += (S)vals[2 * k + 1].x;
            b += (S)vals[2 * k + 1].y;
        }
    }
    if (DT == IN_U8 || DT == IN_U16) {
        a = (S)fa;
        b = (S)fb;
    }
    *sa = a;
    *sb = b;
}

// The subtracted level of one A-scan: its mean rounded to an integer for
// integer samples (so x - c is exact in float), the plain mean for float input.
OPE_HD float split_level(double total, int n, bool integer) {
    const double m = total / (double)n;
    return integer ? (float)std::rint(m) : (float)m;
}

// Step C: write spec = x - c with replicated edges.
template <int N>
OPE_HD void phase_split_store(int t, const float2* vals, float2 c, float2* spec) {
    constexpr int T = Plan<N>::T;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int p = t + k * T;
        const float2 v0 = sub2(vals[2 * k], c), v1 = sub2(vals[2 * k + 1], c);
        OPE_SMEM_CHECK(SPEC_PAD + 2 * p + 1 < N + 2 * SPEC_PAD);
        *reinterpret_cast<float4*>(&spec[SPEC_PAD + 2 * p]) = make_float4(v0.x, v0.y, v1.x, v1.y);
        if (p == 0)
            for (int e = 0; e < SPEC_PAD; ++e) spec[e] = v0;
        if (p == N / 2 - 1)
            for (int e = 0; e < SPEC_PAD; ++e) spec[SPEC_PAD + N + e] = v1;
    }
}

// ------------------------------------------ packed integer spectrum (8/16-bit) --
// For 8- and 16-bit samples without rolling-average DC removal the unpacked
// spectrum is kept as integers: one 32-bit word per sample holds the pair's
// two raw samples (row a in the low half, row b in the high half), half the
// bytes of the float pair. A tap is converted in registers exactly:
// (2^23 + u) - (2^23 + c) = u - c, the same float as the float spectrum holds.

// The pair (2^23 + u_a, 2^23 + u_b) of a packed word: exact floats, no arithmetic.
OPE_HD float2 packed_biased(uint32_t w) {
#if defined(__CUDA_ARCH__)
    const float lo = __uint_as_float(__byte_perm(w, 0x4B00u, 0x5410));
    const float hi = __uint_as_float(__byte_perm(w, 0x4B00u, 0x5432));
#else
    const float lo = bits_f(static_cast<int>(0x4B000000u | (w & 0xFFFFu)));
    const float hi = bits_f(static_cast<int>(0x4B000000u | (w >> 16)));
#endif
    return make_float2(lo, hi);
}

OPE_HD float2 packed_to_pair(uint32_t w, float2 cbias) { return sub2(packed_biased(w), cbias); }

// Samples 2p and 2p+1 of both rows as packed words; adds them to the row sums.
template <int DT>
OPE_HD void load_pos2_packed(const unsigned char* stage, int n, int p, uint32_t* w, int* sa, int* sb) {
    using raw_t = typename InTraits<DT>::raw_t;
    const raw_t* ra = reinterpret_cast<const raw_t*>(stage);
    const raw_t* rb = ra + n;
    uint32_t a0, a1, b0, b1;
#if defined(__CUDA_ARCH__)
    if (DT == IN_U16) {
        const uint32_t wa = *reinterpret_cast<const uint32_t*>(ra + 2 * p);
        const uint32_t wb = *reinterpret_cast<const uint32_t*>(rb + 2 * p);
        w[0] = __byte_perm(wa, wb, 0x5410);
        w[1] = __byte_perm(wa, wb, 0x7632);
        *sa += (int)(wa & 0xFFFFu) + (int)(wa >> 16);
        *sb += (int)(wb & 0xFFFFu) + (int)(wb >> 16);
        return;
    }
#endif
    a0 = ra[2 * p];
    a1 = ra[2 * p + 1];
    b0 = rb[2 * p];
    b1 = rb[2 * p + 1];
    w[0] = a0 | (b0 << 16);
    w[1] = a1 | (b1 << 16);
    *sa += (int)(a0 + a1);
    *sb += (int)(b0 + b1);
}

// Step A of the packed path: thread t packs the sample pairs p = t + k*T
// (k < 8) and sums each row (exact integers).
template <int N, int DT>
OPE_HD void phase_split_load_packed(int t, const unsigned char* stage, uint32_t* words, int* sa, int* sb) {
    constexpr int T = Plan<N>::T;
    int a = 0, b = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) load_pos2_packed<DT>(stage, N, t + k * T, words + 2 * k, &a, &b);
    *sa = a;
    *sb = b;
}

// Step C of the packed path: the words into the spectrum with replicated edges.
template <int N>
OPE_HD void phase_store_packed(int t, const uint32_t* words, uint32_t* specw) {
    constexpr int T = Plan<N>::T;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int p = t + k * T;
        OPE_SMEM_CHECK(SPEC_PAD + 2 * p + 1 < N + 2 * SPEC_PAD);
#if defined(__CUDA_ARCH__)
        *reinterpret_cast<uint2*>(&specw[SPEC_PAD + 2 * p]) = make_uint2(words[2 * k], words[2 * k + 1]);
#else
        specw[SPEC_PAD + 2 * p] = words[2 * k];
        specw[SPEC_PAD + 2 * p + 1] = words[2 * k + 1];
#endif
        if (p == 0)
            for (int e = 0; e < SPEC_PAD; ++e) specw[e] = words[0];
        if (p == N / 2 - 1)
            for (int e = 0; e < SPEC_PAD; ++e) specw[SPEC_PAD + N + e] = words[2 * k + 1];
    }
}

// DataParameters::bitshift as the reference's GPU path applies it
// (inputToCufftComplex_and_bitshift, cuda_kernels.cu:45-63; the reference CPU
// backend ignores the flag): every 8- or 16-bit sample shifted right by 4,
// in place in the stage before the unpack, so every later step sees the
// shifted integers.
template <int N, int DT>
OPE_HD void phase_bitshift(int t, unsigned char* stage) {
    using raw_t = typename InTraits<DT>::raw_t;
    constexpr int T = Plan<N>::T;
    constexpr int WORDS = 2 * N * (int)sizeof(raw_t) / 4;  // 32-bit words of the two rows
    const uint32_t mask = DT == IN_U8 ? 0x0F0F0F0Fu : 0x0FFF0FFFu;
    uint32_t* w = reinterpret_cast<uint32_t*>(stage);
    for (int i = t; i < WORDS; i += T) w[i] = (w[i] >> 4) & mask;
}

// Rolling-average DC removal (cpu_kernels.tpp:56-82): x[i] -= mean of
// x[i-(W-1) .. min(i+W, N-1)]. Window sums come from exact integer prefix sums
// (the reference accumulates them in float; for integer input whose running
// sum stays below 2^24 both are identical).
//
// Prefix-sum word w (2*i + row) lives at pfx_idx(w): two pad words per 32 put
// the 16-sample segments of consecutive threads, and the window ends that
// consecutive threads read, in distinct banks, and keep the two rows' entries of
// sample i (words 2i, 2i + 1) one aligned pair, read and written together.
OPE_HD int pfx_idx(int w) { return w + 2 * (w >> 5); }

// The two rows' prefix entries of one sample, as one aligned pair.
template <typename S>
struct PfxPair {
    S a, b;
};

// The 16 samples [16t, 16t+16) of both rows, widened to the sum type (device:
// 16-byte shared loads).
template <int N, int DT>
OPE_HD void load_raw16(const unsigned char* stage, int t, typename InTraits<DT>::sum_t* xa,
                       typename InTraits<DT>::sum_t* xb) {
    using raw_t = typename InTraits<DT>::raw_t;
    using sum_t = typename InTraits<DT>::sum_t;
    const raw_t* ra = reinterpret_cast<const raw_t*>(stage) + 16 * t;
    const raw_t* rb = ra + N;
#if defined(__CUDA_ARCH__)
    constexpr int Q = (int)sizeof(raw_t);  // 16-byte words per 16 samples
    uint4 qa[Q], qb[Q];
#pragma unroll
    for (int w = 0; w < Q; ++w) {
        qa[w] = reinterpret_cast<const uint4*>(ra)[w];
        qb[w] = reinterpret_cast<const uint4*>(rb)[w];
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int e = k * Q;  // byte offset of sample k
        const uint4& wa = qa[e >> 4];
        const uint4& wb = qb[e >> 4];
        const int lane = (e >> 2) & 3;
        const unsigned ua = lane == 0 ? wa.x : lane == 1 ? wa.y : lane == 2 ? wa.z : wa.w;
        const unsigned ub = lane == 0 ? wb.x : lane == 1 ? wb.y : lane == 2 ? wb.z : wb.w;
        if constexpr (DT == IN_U8) {
            xa[k] = (sum_t)((ua >> (8 * (k & 3))) & 0xFFu);
            xb[k] = (sum_t)((ub >> (8 * (k & 3))) & 0xFFu);
        } else if constexpr (DT == IN_U16) {
            xa[k] = (sum_t)((ua >> (16 * (k & 1))) & 0xFFFFu);
            xb[k] = (sum_t)((ub >> (16 * (k & 1))) & 0xFFFFu);
        } else if constexpr (DT == IN_U32) {
            xa[k] = (sum_t)ua;
            xb[k] = (sum_t)ub;
        } else {
            xa[k] = (sum_t)__uint_as_float(ua);
            xb[k] = (sum_t)__uint_as_float(ub);
        }
    }
#else
    for (int k = 0; k < 16; ++k) {
        xa[k] = (sum_t)ra[k];
        xb[k] = (sum_t)rb[k];
    }
#endif
}

// Step A: thread t owns samples [16t, 16t+16); returns its two row totals.
template <int N, int DT>
OPE_HD void phase_dc_local(int t, const unsigned char* stage, typename InTraits<DT>::sum_t* tot_a,
                           typename InTraits<DT>::sum_t* tot_b) {
    using sum_t = typename InTraits<DT>::sum_t;
    sum_t xa[16], xb[16];
    load_raw16<N, DT>(stage, t, xa, xb);
    sum_t sa = 0, sb = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        sa += xa[k];
        sb += xb[k];
    }
    *tot_a = sa;
    *tot_b = sb;
}

// Step B: with the exclusive prefix of the totals, write prefix sums
// P_row(i) = sum_{k < i} x_row[k] for i in [16t, 16t+16] (P(0) = 0) to word
// pfx_idx(2*i + row).
template <int N, int DT>
OPE_HD void phase_dc_prefix(int t, const unsigned char* stage, typename InTraits<DT>::sum_t ex_a,
                            typename InTraits<DT>::sum_t ex_b, typename InTraits<DT>::sum_t* pfx) {
    using sum_t = typename InTraits<DT>::sum_t;
    sum_t xa[16], xb[16];
    load_raw16<N, DT>(stage, t, xa, xb);
    sum_t sa = ex_a, sb = ex_b;
    if (t == 0) {
        pfx[pfx_idx(0)] = 0;
        pfx[pfx_idx(1)] = 0;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const int i = 16 * t + k;
        sa += xa[k];
        sb += xb[k];
        OPE_SMEM_CHECK(pfx_idx(2 * (i + 1) + 1) < pfx_idx(2 * (N + 1)));
        *reinterpret_cast<PfxPair<sum_t>*>(&pfx[pfx_idx(2 * (i + 1))]) = PfxPair<sum_t>{sa, sb};
    }
}

// Rolling-average DC removal in the reference's own order
// (rollingAverageDCRemoval, cpu_kernels.tpp:56-82): one sequential float
// prefix sum per A-scan, cs[i+1] = cs[i] + x[i], each addition rounded. The
// chain of additions is serial, so threads 0 and 1 run the two rows' sums
// (row t) while the team waits; entry i of row r lives at pfx_idx(2*i + r).
template <int DT>
OPE_HD float sample_as_float(const unsigned char* stage, int n, int row, int i) {
    using raw_t = typename InTraits<DT>::raw_t;
    const raw_t x = reinterpret_cast<const raw_t*>(stage)[row * n + i];
    if (DT == IN_U32) {
#if defined(__CUDA_ARCH__)
        return __uint2float_rn((unsigned)x);
#else
        return (float)(unsigned)x;
#endif
    }
    return (float)x;
}

// Whether a row total of non-negative integer samples keeps every partial sum
// of a float prefix exact (below 2^24).
template <typename S>
OPE_HD bool dc_prefix_exact_in_float(S total) { return total < (S)16777216; }

// The samples are read in chunks of 32 into registers before the chunk's 32
// dependent additions: the prefix stores go to shared memory too, so a load
// after a store could not be issued ahead of it, and each step would wait
// out a shared-memory round trip instead of one addition.
template <int N, int DT>
OPE_HD void phase_dc_ref_scan(int t, const unsigned char* stage, float* pf) {
    if (t > 1) return;
    constexpr int C = 32;
    static_assert(N % C == 0, "whole chunks");
    float s = 0.0f;
    pf[pfx_idx(t)] = 0.0f;
#pragma unroll 1
    for (int i0 = 0; i0 < N; i0 += C) {
        float xs[C];
#pragma unroll
        for (int k = 0; k < C; ++k) xs[k] = sample_as_float<DT>(stage, N, t, i0 + k);
#pragma unroll
        for (int k = 0; k < C; ++k) {
            s = fadd_rn(s, xs[k]);
            OPE_SMEM_CHECK(pfx_idx(2 * (i0 + k + 1) + t) < pfx_idx(2 * (N + 1)));
            pf[pfx_idx(2 * (i0 + k + 1) + t)] = s;
        }
    }
}

// ------------------------ reference-order prefix of 16-bit samples in parallel --
// The same sequential float prefix, cs[i+1] = fl(cs[i] + x[i]), evaluated by the
// team instead of one thread per row, bit for bit. It rests on two facts about
// adding integer samples x to a non-negative float prefix s:
//  * below 2^24 every partial sum is an exact integer;
//  * in a binade [2^k, 2^(k+1)) with k >= 24 every float is a multiple of
//    u = 2^(k-23), and fl(s + x) rounds s/u + x/u to the nearest integer,
//    ties to even, so the increment in units of u depends only on x and on the
//    parity of s/u. A run of samples therefore adds the same number of ulps to
//    every start in the binade with the same parity, as long as no partial
//    result reaches 2^(k+1).
// Segments are 64 samples of one row, split into four 16-sample parts. Step 1:
// each segment's four threads build step records (refpar_step) for its parts in
// the binade of the row's exact integer prefix at the segment start and in the
// next binade, with the float additions from synthetic starts, and compose the
// first set into the whole segment's record. Step 2: threads 0 and 32 walk their
// row's segments in order from 0, one record per segment; a segment whose record
// does not apply (it crosses 2^24 or a binade boundary, or the walk's value lies
// in another binade than the exact prefix) is walked part by part, and only a
// part that itself crosses is added sample by sample. The walk's value is the
// prefix as an exact integer (every float below 2^30 is one). Step 3: the four
// threads write the segment's 64 prefix entries from its start value with the
// float additions, i.e. exactly the entries of the sequential sum.
constexpr int REFPAR_SEG = 64;

OPE_HD int refpar_binade(unsigned v) {  // floor(log2 v), v > 0
#if defined(__CUDA_ARCH__)
    return 31 - __clz((int)v);
#else
    int k = 0;
    while (v >> (k + 1)) ++k;
    return k;
#endif
}

OPE_HD unsigned refpar_f2u(float f) {  // an exact integer-valued float < 2^32
#if defined(__CUDA_ARCH__)
    return __float2uint_rn(f);
#else
    return (unsigned)f;
#endif
}

OPE_HD float refpar_u2f(unsigned v) {  // exact for the prefix values (floats below 2^29)
#if defined(__CUDA_ARCH__)
    return __uint2float_rn(v);
#else
    return (float)v;
#endif
}

// Samples [8k, 8k + 8) of segment q of row `row` as exact floats, read as one
// 16-byte word. On the device each float is 2^23 + x, built by a byte permute,
// minus 2^23 (exact): conversion instructions run at a fraction of the FP32
// rate, and the few threads of a segment step would spend most of their time
// in them.
template <int N>
OPE_HD void refpar_load8(const unsigned char* stage, int row, int q, int k, float* x) {
    const unsigned short* p = reinterpret_cast<const unsigned short*>(stage) + row * N + REFPAR_SEG * q + 8 * k;
#if defined(__CUDA_ARCH__)
    const uint4 w = *reinterpret_cast<const uint4*>(p);
    const unsigned v[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        x[2 * j] = fsub_rn(__uint_as_float(__byte_perm(v[j], 0x4B00u, 0x5410)), 8388608.0f);
        x[2 * j + 1] = fsub_rn(__uint_as_float(__byte_perm(v[j], 0x4B00u, 0x5432)), 8388608.0f);
    }
#else
    for (int j = 0; j < 8; ++j) x[j] = (float)p[j];
#endif
}

// A step record {hi, u, d0 * u, d1 * u}: for a prefix value s (an exact
// integer) with u << 23 <= s < hi, the run of samples takes s to s + d0 * u if
// s / u is even and to s + d1 * u if it is odd. For a binade k >= 24, u = 2^(k-23)
// and hi = 2^(k+1) - (the run's exact sum) - (its roundings' bound): the run
// stays in the binade. For the exact zone u = 0, hi = 2^24 - sum + 1 and
// d0 = d1 = sum: every partial sum stays an exact integer.
OPE_HD bool refpar_step(unsigned& s, int4 g) {
    const unsigned u = (unsigned)g.y;
    if (s < (u << 23) || s >= (unsigned)g.x) return false;
    s += (unsigned)((s & u) ? g.w : g.z);
    return true;
}

// Record of a run with exact sum `sum`, in binade k (k < 24: the exact zone),
// from its increments d0, d1 (in ulps) and the run's length in samples.
OPE_HD int4 refpar_record(int k, unsigned sum, int d0, int d1, int len) {
    if (k < 24) return make_int4((int)((1u << 24) - sum + 1u), 0, (int)sum, (int)sum);
    const int sh = k - 23;
    const unsigned u = 1u << sh;
    return make_int4((int)((2u << k) - sum - (unsigned)(len / 2) * u), (int)u, d0 << sh, d1 << sh);
}

// Shared-memory areas of the three steps (in the spectrum area, which the
// window-mean step writes last): per (segment q, row r), index 2q + r, the
// segment's record for the binade of its exact prefix; the records of its four
// 16-sample parts for that binade and for the next one (8 per index); and the
// segment's start value.
template <int N>
struct RefparArea {
    static constexpr int NSEG = N / REFPAR_SEG;
    int4* seg;
    int4* part;
    unsigned* start;
    OPE_HD explicit RefparArea(unsigned char* base)
        : seg(reinterpret_cast<int4*>(base)),
          part(reinterpret_cast<int4*>(base) + 2 * NSEG),
          start(reinterpret_cast<unsigned*>(reinterpret_cast<int4*>(base) + 2 * NSEG * 9)) {}
    static constexpr int BYTES = 2 * NSEG * (9 * 16 + 4);
};

// Step 1. Segment q's four threads 4q .. 4q+3: thread 4q + 2r + b builds, for
// row r, the records of the segment's four 16-sample parts in binade k + b, k the
// binade of the row's exact prefix at the segment start (ex_a / ex_b: the values
// thread 4q holds after the team scan; the exact zone counts as binade 23, its
// next one is 24), with the float additions from the starts 2^k' and 2^k' + u of
// that binade; the b = 0 thread also composes them into the whole segment's record.
template <int N>
OPE_HD void phase_dc_refpar_seg(int t, const unsigned char* stage, int ex_a, int ex_b, unsigned char* area) {
    static_assert(N % REFPAR_SEG == 0 && 4 * (N / REFPAR_SEG) <= N / 16, "four threads per 64-sample segment");
    const RefparArea<N> A(area);
    const int q = t >> 2, r = (t >> 1) & 1, b = t & 1;
    const unsigned ex = (unsigned)(r ? ex_b : ex_a);
    const int k0 = ex >= (1u << 24) ? refpar_binade(ex) : 23;
    const int k = k0 + b;
    const int sh = k - 23;
    const unsigned base = 1u << k;
    const float s0_init = refpar_u2f(base), s1_init = refpar_u2f(base + (1u << sh));
    int d0[4], d1[4];
    unsigned sums[4];
    int4* part = A.part + 8 * (2 * q + r);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float x[16];
        refpar_load8<N>(stage, r, q, 2 * j, x);
        refpar_load8<N>(stage, r, q, 2 * j + 1, x + 8);
        float s0 = s0_init, s1 = s1_init, sum = 0.0f;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            s0 = fadd_rn(s0, x[i]);
            s1 = fadd_rn(s1, x[i]);
            sum = fadd_rn(sum, x[i]);  // exact: below 2^24
        }
        sums[j] = refpar_f2u(sum);
        d0[j] = (int)((refpar_f2u(s0) - base) >> sh);
        d1[j] = (int)((refpar_f2u(s1) - base - (1u << sh)) >> sh);
        part[2 * j + b] = refpar_record(k, sums[j], d0[j], d1[j], 16);
    }
    if (b == 0) {
        // the parts composed: the parity after a part of d ulps flips with d's parity
        int inc[2];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            int acc = 0, par = p;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int d = par ? d1[j] : d0[j];
                acc += d;
                par ^= d & 1;
            }
            inc[p] = acc;
        }
        OPE_SMEM_CHECK(2 * q + r < 2 * (N / REFPAR_SEG));
        A.seg[2 * q + r] = refpar_record(k, sums[0] + sums[1] + sums[2] + sums[3], inc[0], inc[1], REFPAR_SEG);
    }
}

// The float additions of samples [16j, 16j + 16) of segment q of row `row` onto f.
template <int N>
OPE_HD float refpar_add_part(const unsigned char* stage, int row, int q, int j, float f) {
    float x[16];
    refpar_load8<N>(stage, row, q, 2 * j, x);
    refpar_load8<N>(stage, row, q, 2 * j + 1, x + 8);
#pragma unroll
    for (int i = 0; i < 16; ++i) f = fadd_rn(f, x[i]);
    return f;
}

// A segment whose record does not apply (it crosses 2^24 or a binade boundary,
// or the walk's value is not in the binade of the exact prefix): its four parts,
// each by its record for the segment's binade or the next one, or, for the part
// that crosses, by its 16 float additions.
template <int N>
OPE_HD unsigned refpar_walk_parts(const unsigned char* stage, const int4* part, int row, int q, unsigned s) {
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
        if (refpar_step(s, part[2 * j]) || refpar_step(s, part[2 * j + 1])) continue;
        s = refpar_f2u(refpar_add_part<N>(stage, row, q, j, refpar_u2f(s)));
    }
    return s;
}

#if defined(__CUDA_ARCH__)
// Consecutive segment records of one binade composed: from a start s with
// u << 23 <= s < hi, an even s / u adds a, an odd one adds b.
struct RefparComp {
    unsigned hi, a, b;
};

// f first, then g (one u). After f the parity of s / u flips with that of the
// ulps f added; the composite's bound keeps both parts valid (conservatively,
// with the larger of f's increments).
__device__ __forceinline__ RefparComp refpar_compose(RefparComp f, RefparComp g, unsigned u) {
    RefparComp c;
    c.a = f.a + ((f.a & u) ? g.b : g.a);
    c.b = f.b + ((f.b & u) ? g.a : g.b);
    const unsigned m = f.a > f.b ? f.a : f.b;
    const unsigned gh = g.hi > m ? g.hi - m : 0u;
    c.hi = f.hi < gh ? f.hi : gh;
    return c;
}

__device__ __forceinline__ RefparComp refpar_shfl_up(RefparComp c, int d) {
    return RefparComp{__shfl_up_sync(0xffffffffu, c.hi, d), __shfl_up_sync(0xffffffffu, c.a, d),
                      __shfl_up_sync(0xffffffffu, c.b, d)};
}

// One warp walks row r, 32 segments at a time, lane L holding segment L's
// record. Runs of consecutive segments in one binade (one u) are composed by a
// segmented scan over the lanes; the walk then takes a whole run at once: every
// lane of the run forms its start value from the run's start and the composite
// of the run's earlier segments. From the first lane whose composite or own
// record does not apply (normally a run's last segment, where the walk crosses
// into the next binade), the segments of that run are walked one at a time,
// part by part where needed. Every lane keeps the same walk value, so the warp
// never diverges.
template <int N>
__device__ __forceinline__ void refpar_walk_scan(int lane, int r, const unsigned char* stage,
                                                 const RefparArea<N>& A) {
    constexpr int NSEG = RefparArea<N>::NSEG;
    constexpr int M = (NSEG + 31) / 32;
    constexpr int J = NSEG < 32 ? NSEG : 32;  // segments per block of lanes
    constexpr unsigned LIVE = J == 32 ? 0xffffffffu : ((1u << J) - 1u);
    unsigned s = 0;
#pragma unroll 1
    for (int m = 0; m < M; ++m) {
        const int q = 32 * m + lane;
        const int4 g = lane < J ? A.seg[2 * q + r] : make_int4(0, 0, 0, 0);
        const unsigned u = (unsigned)g.y;
        const unsigned uprev = __shfl_up_sync(0xffffffffu, u, 1);
        const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || u != uprev) & LIVE;
        const int rs = 31 - __clz((int)(heads & (0xffffffffu >> (31 - lane))));  // this lane's run start
        RefparComp c{(unsigned)g.x, (unsigned)g.z, (unsigned)g.w};
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const RefparComp o = refpar_shfl_up(c, d);
            if (lane - d >= rs) c = refpar_compose(o, c, u);
        }
        const RefparComp ex = refpar_shfl_up(c, 1);  // the run's segments before this lane
        int L = 0;
        while (L < J) {
            if ((heads >> L) & 1u) {
                const unsigned later = heads & ~((2u << L) - 1u);
                const int end = later ? __ffs((int)later) - 1 : J;
                const bool in = lane >= L && lane < end;
                unsigned my = s;
                bool ok = s >= (u << 23);
                if (lane > L) {
                    ok = ok && s < ex.hi;
                    my = s + ((s & u) ? ex.b : ex.a);
                }
                ok = ok && my < (unsigned)g.x;
                const unsigned bad = __ballot_sync(0xffffffffu, in && !ok);
                const int stop = bad ? __ffs((int)bad) - 1 : end;
                if (lane >= L && lane < stop) A.start[2 * q + r] = my;
                if (stop > L) s = __shfl_sync(0xffffffffu, my + ((my & u) ? (unsigned)g.w : (unsigned)g.z), stop - 1);
                L = stop;
                if (stop == end) continue;
            }
            // segment L on its own: its record, else part by part
            const int4 gl = make_int4(__shfl_sync(0xffffffffu, g.x, L), __shfl_sync(0xffffffffu, g.y, L),
                                      __shfl_sync(0xffffffffu, g.z, L), __shfl_sync(0xffffffffu, g.w, L));
            const int ql = 32 * m + L;
            if (lane == 0) A.start[2 * ql + r] = s;
            if (!refpar_step(s, gl)) s = refpar_walk_parts<N>(stage, A.part + 8 * (2 * ql + r), r, ql, s);
            ++L;
        }
    }
}
#endif

// Step 2. Each row's segments in order from 0: one record step per segment; a
// segment whose record does not apply is walked part by part
// (refpar_walk_parts). On the device warp r walks row r by runs
// (refpar_walk_scan; one warp walks both rows in turn when the team is one warp);
// the host walk, one thread per row, gives the same values.
template <int N>
OPE_HD void phase_dc_refpar_walk(int t, const unsigned char* stage, unsigned char* area) {
    const RefparArea<N> A(area);
#if defined(__CUDA_ARCH__)
    const int warp = t >> 5, lane = t & 31;
    if (Plan<N>::T >= 64) {
        if (warp < 2) refpar_walk_scan<N>(lane, warp, stage, A);
    } else {
        refpar_walk_scan<N>(lane, 0, stage, A);
        refpar_walk_scan<N>(lane, 1, stage, A);
    }
#else
    if (t > 1) return;
    const int r = t;
    unsigned s = 0;
    for (int q = 0; q < RefparArea<N>::NSEG; ++q) {
        A.start[2 * q + r] = s;
        if (!refpar_step(s, A.seg[2 * q + r])) s = refpar_walk_parts<N>(stage, A.part + 8 * (2 * q + r), r, q, s);
    }
#endif
}

// Step 3. Segment q's four threads write its prefix entries: thread 4q + 2r + h
// the 32 entries of half h of row r, from the segment's start value (half 1: after
// the first two parts, by their records or their additions), with the float
// additions.
template <int N>
OPE_HD void phase_dc_refpar_fill(int t, const unsigned char* stage, unsigned char* area, float* pf) {
    const RefparArea<N> A(area);
    const int q = t >> 2, r = (t >> 1) & 1, h = t & 1;
    if (t == 0) {
        pf[pfx_idx(0)] = 0.0f;
        pf[pfx_idx(1)] = 0.0f;
    }
    unsigned s0 = A.start[2 * q + r];
    if (h) {
        const int4* part = A.part + 8 * (2 * q + r);
#pragma unroll 1
        for (int j = 0; j < 2; ++j)
            if (!refpar_step(s0, part[2 * j]) && !refpar_step(s0, part[2 * j + 1]))
                s0 = refpar_f2u(refpar_add_part<N>(stage, r, q, j, refpar_u2f(s0)));
    }
    float s = refpar_u2f(s0);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float x[8];
        refpar_load8<N>(stage, r, q, 4 * h + c, x);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int e = REFPAR_SEG * q + 32 * h + 8 * c + i + 1;
            s = fadd_rn(s, x[i]);
            OPE_SMEM_CHECK(pfx_idx(2 * e + r) < pfx_idx(2 * (N + 1)));
            pf[pfx_idx(2 * e + r)] = s;
        }
    }
}

// Step C: subtract the window means and write the spectrum pairs. A window of
// a power-of-two count (the interior, when 2W is one: W = 64 by default) is
// divided by multiplying with its exact reciprocal, which equals the correctly
// rounded quotient; other counts use the correctly rounded division.
// REF = false: exact window sums from the integer prefix sums of
// phase_dc_prefix; REF = true: the reference's float difference of two entries
// of the sequential float prefix sum (phase_dc_ref_scan).
//
// Chunks of 8 samples whose windows all hold 2W samples (the interior), when 2W
// is a power of two, take a short path: both rows' prefix entries of a window
// end as one pair, the two window sums and means as float pairs, and for 8/16-bit
// samples whose window sums stay below 2^23 the sums converted exactly as
// (2^23 + S) - 2^23 (the bits of 2^23 + S are those of 2^23 with S in the
// mantissa) instead of by conversion instructions. Same values as the general
// path: the sums are exact integers below 2^24 either way, and the products with
// 1/(2W) are exact.
template <int N, int DT, bool REF = false>
OPE_HD void phase_dc_apply(int t, const unsigned char* stage, const void* pfx_v, int W, float2* spec) {
    using sum_t = typename InTraits<DT>::sum_t;
    constexpr int T = Plan<N>::T;
    const int full = 2 * W;
    const bool full_pow2 = (full & (full - 1)) == 0;
    const float full_inv = 1.0f / (float)full;  // exact when full is a power of two
    constexpr int MAXV = DT == IN_U8 ? 255 : 65535;
    const bool bias_sum = (DT == IN_U8 || DT == IN_U16) && (long long)full * MAXV < 8388608LL;
    // not unrolled: two copies of the chunk body cost more in instruction
    // fetch than the loop (measured: 90 against 107 M A-scans/s at N = 2048)
#pragma unroll 1
    for (int c = t; c < N / 8; c += T) {
        float2 v[8];
        load_chunk8<DT>(stage, N, c, v);
        if (full_pow2 && 8 * c >= W - 1 && 8 * c + 7 + W < N - 1) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int i = 8 * c + k;
                const int hi = pfx_idx(2 * (i + W + 1)), lo = pfx_idx(2 * (i - W + 1));
                float2 sum;
                if constexpr (REF) {
                    const float* pf = static_cast<const float*>(pfx_v);
                    sum = sub2(*reinterpret_cast<const float2*>(&pf[hi]), *reinterpret_cast<const float2*>(&pf[lo]));
                } else {
                    const sum_t* pfx = static_cast<const sum_t*>(pfx_v);
                    const PfxPair<sum_t> ph = *reinterpret_cast<const PfxPair<sum_t>*>(&pfx[hi]);
                    const PfxPair<sum_t> pl = *reinterpret_cast<const PfxPair<sum_t>*>(&pfx[lo]);
                    const sum_t da = ph.a - pl.a, db = ph.b - pl.b;
                    if (bias_sum)
                        sum = sub2(make_float2(bits_f((int)(0x4B000000u | (unsigned)da)),
                                               bits_f((int)(0x4B000000u | (unsigned)db))),
                                   dup2(8388608.0f));
                    else
                        sum = make_float2((float)da, (float)db);
                }
                v[k] = sub2(v[k], mul2(sum, dup2(full_inv)));
            }
        } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            int i = 8 * c + k;
            int start = (i >= W - 1) ? i - (W - 1) : 0;
            int end = (i + W < N - 1) ? i + W : N - 1;
            float fa, fb;
            if constexpr (REF) {
                const float* pf = static_cast<const float*>(pfx_v);
                fa = fsub_rn(pf[pfx_idx(2 * (end + 1))], pf[pfx_idx(2 * start)]);
                fb = fsub_rn(pf[pfx_idx(2 * (end + 1) + 1)], pf[pfx_idx(2 * start + 1)]);
            } else {
                const sum_t* pfx = static_cast<const sum_t*>(pfx_v);
                fa = (float)(pfx[pfx_idx(2 * (end + 1))] - pfx[pfx_idx(2 * start)]);
                fb = (float)(pfx[pfx_idx(2 * (end + 1) + 1)] - pfx[pfx_idx(2 * start + 1)]);
            }
            const int n = end - start + 1;
            float ma, mb;
            if (full_pow2 && n == full) {
                ma = fmul_rn(fa, full_inv);
                mb = fmul_rn(fb, full_inv);
            } else {
                float cnt = (float)n;
#if defined(__CUDA_ARCH__)
                ma = __fdiv_rn(fa, cnt);
                mb = __fdiv_rn(fb, cnt);
#else
                ma = fa / cnt;
                mb = fb / cnt;
#endif
            }
            v[k] = sub2(v[k], make_float2(ma, mb));
        }
        }
#pragma unroll
        for (int i = 0; i < 8; i += 2)
            *reinterpret_cast<float4*>(&spec[SPEC_PAD + 8 * c + i]) =
                make_float4(v[i].x, v[i].y, v[i + 1].x, v[i + 1].y);
        if (c == 0)
            for (int k = 0; k < SPEC_PAD; ++k) spec[k] = v[0];
        if (c == N / 8 - 1)
            for (int k = 0; k < SPEC_PAD; ++k) spec[SPEC_PAD + N + k] = v[7];
    }
}

// ------------------------------------------------- resample, window, phase --
// Produces the pass-0 inputs v[s] = z(t + s*T), s < 16.
template <int N, int INTERP>
OPE_HD void phase_prestage(int t, const float2* spec, const ChainArgs& a, cp* v) {
    constexpr int T = Plan<N>::T;
    const float2 NZ = dup2(a.neg_zero);
#pragma unroll
    for (int s = 0; s < 16; ++s) {
        const int j = t + s * T;
        float2 y;
        if (INTERP == INTERP_NONE) {
            y = spec[SPEC_PAD + j];
        } else if (INTERP == INTERP_LINEAR) {
            // kLinearizationLinear (cpu_kernels.tpp:95-110): y1 + (y2 - y1) * (nx - n1)
            int2 e = a.lin[j];
            OPE_SMEM_CHECK(e.x >= 0 && e.x + 1 < N + 2 * SPEC_PAD);
            float2 y1 = spec[e.x];
            float2 y2 = spec[e.x + 1];
            const float fr = bits_f(e.y);
            y = add2(y1, mul2x(sub2(y2, y1), dup2(fr), NZ));
        } else if (INTERP == INTERP_CUBIC) {
            // kLinearizationCubic + cubicHermiteInterpolation (cpu_kernels.tpp:124-145,486-502)
#if defined(__CUDA_ARCH__)
            const int2 e = __ldg(a.cub + j);
#else
            const int2 e = a.cub[j];
#endif
            const int i0 = e.x & 0xFFFF, i1 = (unsigned)e.x >> 16;
            OPE_SMEM_CHECK(i0 < N + 2 * SPEC_PAD && i1 + 2 < N + 2 * SPEC_PAD);
            const float pos = bits_f(e.y), pos2 = fmul_rn(pos, pos);
            float2 y0 = spec[i0], y1 = spec[i1], y2 = spec[i1 + 1], y3 = spec[i1 + 2];
            float2 ca = add2(sub2(mul2x(dup2(3.0f), sub2(y1, y2), NZ), y0), y3);
            float2 cb = sub2(add2(sub2(mul2x(dup2(2.0f), y0, NZ), mul2x(dup2(5.0f), y1, NZ)),
                                  mul2x(dup2(4.0f), y2, NZ)),
                             y3);
            float2 cc = sub2(y2, y0);
            float2 in = add2(add2(mul2x(ca, dup2(pos2), NZ), mul2x(cb, dup2(pos), NZ)), cc);
            y = add2(mul2x(dup2(fmul_rn(0.5f, pos)), in, NZ), y1);
        } else {
            // kLinearizationLanczos (cpu_kernels.tpp:176-195): sequential 16-tap sum
            int b = a.lz_base[j];
            OPE_SMEM_CHECK(b >= 0 && b + 15 < N + 2 * SPEC_PAD);
            float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int k = 0; k < 16; ++k) {
#if defined(__CUDA_ARCH__)
                float w = __ldg(a.lz_w + k * N + j);
#else
                float w = a.lz_w[k * N + j];
#endif
                acc = add2(acc, mul2x(spec[b + k], dup2(w), NZ));
            }
            y = acc;
        }
#if !defined(__CUDA_ARCH__)
        if (a.resampled_out) {  // CPU emulation only: the k-linearised spectrum of this pair
            a.resampled_out[(long long)j * 2] = y.x;
            a.resampled_out[(long long)j * 2 + 1] = y.y;
        }
#endif
        // applyWindow then dispersionCompensation (cpu_kernels.tpp:198-235):
        // re = y*w*cos, im = y*w*sin with the window folded into the phase
        // factors (w*cos, w*sin), evaluated in double and rounded once and
        // shared by both lanes.
#if defined(__CUDA_ARCH__)
        const float2 q = __ldg(a.wph + j);
#else
        const float2 q = a.wph[j];
#endif
        v[s] = cpmake(mul2x(y, dup2(q.x), NZ), mul2x(y, dup2(q.y), NZ));
    }
}

// phase_prestage on the packed integer spectrum: the same interpolation and
// window-phase arithmetic on the same (exactly converted) tap values.
template <int N, int INTERP>
OPE_HD void phase_prestage_packed(int t, const uint32_t* specw, float2 cbias, const ChainArgs& a, cp* v) {
    constexpr int T = Plan<N>::T;
    const float2 NZ = dup2(a.neg_zero);
#pragma unroll
    for (int s = 0; s < 16; ++s) {
        const int j = t + s * T;
        float2 y;
        if (INTERP == INTERP_NONE) {
            y = packed_to_pair(specw[SPEC_PAD + j], cbias);
        } else if (INTERP == INTERP_LINEAR) {
#if defined(__CUDA_ARCH__)
            const int2 e = __ldg(a.lin + j);
#else
            const int2 e = a.lin[j];
#endif
            OPE_SMEM_CHECK(e.x >= 0 && e.x + 1 < N + 2 * SPEC_PAD);
            // y2 - y1 is the exact difference of the biased taps
            const float2 Y1 = packed_biased(specw[e.x]);
            const float2 d = sub2(packed_biased(specw[e.x + 1]), Y1);
            y = add2(sub2(Y1, cbias), mul2x(d, dup2(bits_f(e.y)), NZ));
        } else if (INTERP == INTERP_CUBIC) {
#if defined(__CUDA_ARCH__)
            const int2 e = __ldg(a.cub + j);
#else
            const int2 e = a.cub[j];
#endif
            const int i0 = e.x & 0xFFFF, i1 = (unsigned)e.x >> 16;
            OPE_SMEM_CHECK(i0 < N + 2 * SPEC_PAD && i1 + 2 < N + 2 * SPEC_PAD);
            const float pos = bits_f(e.y), pos2 = fmul_rn(pos, pos);
            // cubicHermiteInterpolation (cpu_kernels.tpp:486-502) on integer taps
            // y_k = u_k - c: its a, b, c are integers below 2^20, exact in any
            // evaluation order, so they are formed from differences of the
            // biased taps Y_k = 2^23 + u_k (exact, no conversion); with
            // na = -a, fl(a pos^2) = -fl(na pos^2), so the reference's
            // ((a pos^2 + b pos) + c) is (b pos - na pos^2) + c, bit for bit.
            const float2 Y0 = packed_biased(specw[i0]), Y1 = packed_biased(specw[i1]);
            const float2 Y2 = packed_biased(specw[i1 + 1]), Y3 = packed_biased(specw[i1 + 2]);
            const float2 e0 = sub2(Y0, Y1), e2 = sub2(Y2, Y1), e3 = sub2(Y1, Y3);
            const float2 na = fma2(dup2(3.0f), e2, add2(e0, e3));      // y0 - 3(y1 - y2) - y3
            const float2 cb = fma2(dup2(2.0f), e0, fma2(dup2(4.0f), e2, e3));  // 2y0 - 5y1 + 4y2 - y3
            const float2 cc = sub2(e2, e0);                            // y2 - y0
            const float2 in = add2(sub2(mul2x(cb, dup2(pos), NZ), mul2x(na, dup2(pos2), NZ)), cc);
            y = add2(mul2x(dup2(fmul_rn(0.5f, pos)), in, NZ), sub2(Y1, cbias));
        } else {
            const int b = a.lz_base[j];
            OPE_SMEM_CHECK(b >= 0 && b + 15 < N + 2 * SPEC_PAD);
            float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int k = 0; k < 16; ++k) {
#if defined(__CUDA_ARCH__)
                const float w = __ldg(a.lz_w + k * N + j);
#else
                const float w = a.lz_w[k * N + j];
#endif
                acc = add2(acc, mul2x(packed_to_pair(specw[b + k], cbias), dup2(w), NZ));
            }
            y = acc;
        }
#if !defined(__CUDA_ARCH__)
        if (a.resampled_out) {  // CPU emulation only: the k-linearised spectrum of this pair
            a.resampled_out[(long long)j * 2] = y.x;
            a.resampled_out[(long long)j * 2 + 1] = y.y;
        }
#endif
#if defined(__CUDA_ARCH__)
        const float2 q = __ldg(a.wph + j);
#else
        const float2 q = a.wph[j];
#endif
        v[s] = cpmake(mul2x(y, dup2(q.x), NZ), mul2x(y, dup2(q.y), NZ));
    }
}

// ------------------------------------------------------------- FFT passes --
// Stockham pass p with radix R and span NS (the product of the earlier
// radices): DFT d = t + i*T (i < D = 16/R) reads x[d + r*N/R] = slot
// s = i + r*D, multiplies by W_{NS R}^{r k} (k = d mod NS), and writes output
// q to (d - k)*R + k + q*NS.
//
// Radix schedule S: every pass has radix 16 except one of radix LASTR
// (N = 16^(NPASS-1) * LASTR); S = 0 runs that pass last, S >= 1 runs it as
// pass S - 1 (S = 1: first; S = 2: second, e.g. 16*8*16 at N = 2048).
OPE_HD constexpr int short_pass_of(int npass, int s) { return s == 0 ? npass - 1 : s - 1; }

template <int N, int S>
struct Sched {
    static constexpr int NPASS = Plan<N>::NPASS;
    static_assert(S >= 0 && (S == 0 || S - 1 < NPASS), "radix schedule: 0 (short pass last) or 1 + its pass index");
    static constexpr int SHORT = short_pass_of(NPASS, S);
    static constexpr int radix(int p) { return p == SHORT ? Plan<N>::LASTR : 16; }
    static constexpr int span(int p) {
        int v = 1;
        for (int q = 0; q < p; ++q) v *= radix(q);
        return v;
    }
    // Twiddles of pass p >= 1 live in one block of (R-1) x NS entries,
    // entry (r-1)*NS + k = W_{NS*R}^{r*k}: threads with consecutive k read
    // consecutive entries. Blocks of successive passes follow each other.
    static constexpr int tw_off(int p) {
        int o = 0;
        for (int q = 1; q < p; ++q) o += (radix(q) - 1) * span(q);
        return o;
    }
};

template <int N, int P, int S = 0>
struct PassInfo {
    static constexpr int NPASS = Plan<N>::NPASS;
    static constexpr bool LAST = (P == NPASS - 1);
    static constexpr int R = Sched<N, S>::radix(P);
    static constexpr int D = 16 / R;
    static constexpr int NS = Sched<N, S>::span(P);
    static constexpr int TW_SIZE = (P == 0) ? 0 : (R - 1) * NS;
    static constexpr int TW_OFF = Sched<N, S>::tw_off(P);
};

template <int N>
OPE_HD void fft_load(int t, const float4* exch, cp* v) {
    constexpr int T = Plan<N>::T;
#pragma unroll
    for (int s = 0; s < 16; ++s) {
        int e = t + s * T;
        OPE_SMEM_CHECK(xslot(e) < Plan<N>::EXCH_ELEMS);
        float4 q = exch[xslot(e)];
        v[s] = cpmake(make_float2(q.x, q.y), make_float2(q.z, q.w));
    }
}

// FULL = true computes every output of the last pass (all N bins); by default
// the last pass keeps only bins [0, N/2).
template <int N, int P, bool FULL = false, int S = 0>
OPE_HD void fft_twiddle_dft(int t, cp* v, const float2* tw) {
    using PI = PassInfo<N, P, S>;
    constexpr int T = Plan<N>::T;
    constexpr int R = PI::R, D = PI::D, NS = PI::NS;
    constexpr int NOUT = (PI::LAST && !FULL) ? R / 2 : R;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        cp u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = v[i + r * D];
        if (P > 0) {
            const int d = t + i * T;
            const int k = d % NS;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const int idx = PI::TW_OFF + (r - 1) * NS + k;
                OPE_SMEM_CHECK(idx >= 0 && idx < N);
#if defined(__CUDA_ARCH__)
                float2 w = __ldg(tw + idx);
#else
                float2 w = tw[idx];
#endif
                u[r] = cmul_tw(u[r], w.x, w.y);
            }
        }
        if (R == 16) dft16<NOUT>(u);
        else if (R == 8) dft8<NOUT>(u);
        else if (R == 4) dft4v<NOUT>(u);
        else dft2<NOUT>(u);
#pragma unroll
        for (int q = 0; q < NOUT; ++q) v[i + q * D] = u[q];
    }
}

template <int N, int P, int S = 0>
OPE_HD void fft_store(int t, const cp* v, float4* exch) {
    using PI = PassInfo<N, P, S>;
    constexpr int T = Plan<N>::T;
    constexpr int R = PI::R, D = PI::D, NS = PI::NS;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        const int d = t + i * T;
        const int k = d % NS;
        const int base = (d - k) * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            int e = base + q * NS;
            OPE_SMEM_CHECK(e >= 0 && e < N && xslot(e) < Plan<N>::EXCH_ELEMS);
            cp x = v[i + q * D];
            exch[xslot(e)] = make_float4(x.re.x, x.re.y, x.im.x, x.im.y);
        }
    }
}

// ---------------------------------------------------------------- epilogue --
OPE_HD float fast_log2(float x) {
#if defined(__CUDA_ARCH__)
    return __log2f(x);
#else
    return std::log2(x);
#endif
}
OPE_HD float fsqrt(float x) {
#if defined(__CUDA_ARCH__)
    return __fsqrt_rn(x);
#else
    return std::sqrt(x);
#endif
}

// Bin b of the last pass lives in v[i + q*D] for b = (t + i*T) + q*N/R.
template <int N, int S = 0>
struct LastInfo {
    using PI = PassInfo<N, Plan<N>::NPASS - 1, S>;
    static constexpr int R = PI::R, D = PI::D;
    static constexpr int NB = D * (R / 2);  // bins per thread
    OPE_HD static int bin(int t, int i, int q) { return t + i * Plan<N>::T + q * (N / R); }
};

// Adds back the split-off DC level: X[b] += c * dc_resp[b] (both lanes).
OPE_HD cp add_dc(const ChainArgs& a, cp x, int bin, float2 c) {
    if (!a.dc_resp) return x;
#if defined(__CUDA_ARCH__)
    const float2 d = __ldg(a.dc_resp + bin);
#else
    const float2 d = a.dc_resp[bin];
#endif
    return cpmake(fma2(c, dup2(d.x), x.re), fma2(c, dup2(d.y), x.im));
}

// |X|^2 with the optional fixed-pattern subtraction (cpu_kernels.tpp:460-479).
template <int N, int S = 0>
OPE_HD void epi_mag2(int t, const cp* v, const ChainArgs& a, float2 c, float2* mag2) {
    using L = LastInfo<N, S>;
#pragma unroll
    for (int i = 0; i < L::D; ++i)
#pragma unroll
        for (int q = 0; q < L::R / 2; ++q) {
            cp x = add_dc(a, v[i + q * L::D], L::bin(t, i, q), c);
            if (a.fpn) {
                int b = L::bin(t, i, q);
#if defined(__CUDA_ARCH__)
                float2 f = __ldg(a.fpn + b);
#else
                float2 f = a.fpn[b];
#endif
                x.re = sub2(x.re, dup2(f.x));
                x.im = sub2(x.im, dup2(f.y));
            }
            mag2[i * (L::R / 2) + q] = fma2(x.re, x.re, mul2(x.im, x.im));
        }
}

// Output row of A-scan `row`. B-scan flip follows the reference CUDA kernel
// (cuda_kernels.cu:553-573, launched at cuda_backend.cu:690-694): B-scan b is
// mirrored laterally when b is even and b+1 < bscans, i.e. the first B-scan of
// every complete pair; a trailing single B-scan is left as is.
OPE_HD long long out_row(const ChainArgs& a, long long row) {
    if (!a.flip) return row;
    long long bs = row / a.ascans_per_bscan;
    if ((bs & 1) != 0 || bs + 1 >= a.bscans) return row;
    long long in_b = row - bs * a.ascans_per_bscan;
    return bs * a.ascans_per_bscan + (a.ascans_per_bscan - 1 - in_b);
}

}  // namespace ope_b200
