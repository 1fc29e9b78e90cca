// Device-only parts of the fused chain: TMA bulk copies, bounded mbarrier
// waits, team reductions and the persistent __global__ kernel.
#pragma once

#include "chain_kernel.cuh"

namespace ope_b200 {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Non-multicast 1-D bulk copy global -> this CTA's shared memory, completing
// `bytes` of transaction count on `bar`. Source and destination must be
// 16-byte aligned and `bytes` a multiple of 16 (checked by the host).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of `bar`, giving up after timeout_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned long long timeout_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_ns() - t0 > timeout_ns) return false;
    }
    return true;
}

// A team is the group of threads that processes one pair of A-scans.
// CtaTeam: the whole CTA (barrier 0). SubTeam: `count` threads starting at
// thread `base` (both multiples of 32), synchronised by named barrier `id`
// (1..15), so several teams can share one CTA.
struct CtaTeam {
    __device__ __forceinline__ int tid() const { return threadIdx.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};

struct SubTeam {
    int base, id, count;
    __device__ __forceinline__ int tid() const { return (int)threadIdx.x - base; }
    __device__ __forceinline__ void sync() const {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
    }
};

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Exclusive team scan of two values per thread (T threads, T % 32 == 0);
// the team totals too when tot_a / tot_b are given.
template <int T, typename S, class Team>
__device__ __forceinline__ void team_exclusive_scan2(const Team& tm, S& a, S& b, S* scratch, S* tot_a = nullptr,
                                                     S* tot_b = nullptr) {
    const int lane = tm.tid() & 31, warp = tm.tid() >> 5;
    S ia = a, ib = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        S xa = __shfl_up_sync(0xffffffffu, ia, o);
        S xb = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= o) {
            ia += xa;
            ib += xb;
        }
    }
    if (lane == 31) {
        scratch[2 * warp] = ia;
        scratch[2 * warp + 1] = ib;
    }
    tm.sync();
    S pa = 0, pb = 0;
    for (int w = 0; w < warp; ++w) {
        pa += scratch[2 * w];
        pb += scratch[2 * w + 1];
    }
    if (tot_a) {
        S sa = 0, sb = 0;
        for (int w = 0; w < T / 32; ++w) {
            sa += scratch[2 * w];
            sb += scratch[2 * w + 1];
        }
        *tot_a = sa;
        *tot_b = sb;
    }
    a = pa + ia - a;
    b = pb + ib - b;
}

// Team sum of two doubles, in a fixed order (xor butterfly inside each warp,
// then warp totals in warp order) that the CPU emulation reproduces.
template <int T, typename S, class Team>
__device__ __forceinline__ void team_sum2(const Team& tm, S& a, S& b, S* scratch) {
    const int lane = tm.tid() & 31, warp = tm.tid() >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
        scratch[2 * warp] = a;
        scratch[2 * warp + 1] = b;
    }
    tm.sync();
    S ta = 0, tb = 0;
    for (int w = 0; w < T / 32; ++w) {
        ta += scratch[2 * w];
        tb += scratch[2 * w + 1];
    }
    a = ta;
    b = tb;
}

template <int T, class Team>
__device__ __forceinline__ void team_minmax2(const Team& tm, float2& mn, float2& mx, float* scratch) {
    const int lane = tm.tid() & 31, warp = tm.tid() >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn.x = fminf(mn.x, __shfl_xor_sync(0xffffffffu, mn.x, o));
        mn.y = fminf(mn.y, __shfl_xor_sync(0xffffffffu, mn.y, o));
        mx.x = fmaxf(mx.x, __shfl_xor_sync(0xffffffffu, mx.x, o));
        mx.y = fmaxf(mx.y, __shfl_xor_sync(0xffffffffu, mx.y, o));
    }
    if (lane == 0) {
        scratch[4 * warp + 0] = mn.x;
        scratch[4 * warp + 1] = mn.y;
        scratch[4 * warp + 2] = mx.x;
        scratch[4 * warp + 3] = mx.y;
    }
    tm.sync();
    mn = make_float2(scratch[0], scratch[1]);
    mx = make_float2(scratch[2], scratch[3]);
    for (int w = 1; w < T / 32; ++w) {
        mn.x = fminf(mn.x, scratch[4 * w + 0]);
        mn.y = fminf(mn.y, scratch[4 * w + 1]);
        mx.x = fmaxf(mx.x, scratch[4 * w + 2]);
        mx.y = fmaxf(mx.y, scratch[4 * w + 3]);
    }
}

// Output stage for one pair: scaling, affine map, streaming stores.
template <int N, int S, class Team>
__device__ __forceinline__ void epilogue(const Team& tm, int t, const cp* v, const ChainArgs& a, long long row_a,
                                         float2 dc, float* scratch) {
    using L = LastInfo<N, S>;
    constexpr int NB = L::NB;
    float2 mag2[NB];
    epi_mag2<N, S>(t, v, a, dc, mag2);
    float2 res[NB];
    if (a.log_mode) {
#pragma unroll
        for (int k = 0; k < NB; ++k) res[k] = make_float2(fast_log2(mag2[k].x), fast_log2(mag2[k].y));
        if (a.auto_minmax) {
            // logScaleAndTruncate auto range (cpu_kernels.tpp:327-335): per A-scan
            // min/max of 10*log10(|X|^2/(N/2)) over the kept bins.
            const float c10 = 3.01029995663981195214f;  // 10*log10(2)
            const float off = c10 * (float)Plan<N>::LOG2N - c10;  // 10*log10(N/2)
            float2 mn = make_float2(INFINITY, INFINITY), mx = make_float2(-INFINITY, -INFINITY);
#pragma unroll
            for (int k = 0; k < NB; ++k) {
                res[k] = make_float2(fmaf(c10, res[k].x, -off), fmaf(c10, res[k].y, -off));
                mn = make_float2(fminf(mn.x, res[k].x), fminf(mn.y, res[k].y));
                mx = make_float2(fmaxf(mx.x, res[k].x), fmaxf(mx.y, res[k].y));
            }
            // the scratch may lie inside the exchange buffer, which slower
            // threads of the team may still be reading in the last pass
            tm.sync();
            team_minmax2<Plan<N>::T>(tm, mn, mx, scratch);
            float ra = mx.x - mn.x, rb = mx.y - mn.y;
            if (!(ra >= 1e-6f)) ra = 1.0f;
            if (!(rb >= 1e-6f)) rb = 1.0f;
            const float sa = a.mult / ra, sb = a.mult / rb;
#pragma unroll
            for (int k = 0; k < NB; ++k)
                res[k] = make_float2(fmaf(sa, res[k].x - mn.x, a.mult * a.addend),
                                     fmaf(sb, res[k].y - mn.y, a.mult * a.addend));
        } else {
#pragma unroll
            for (int k = 0; k < NB; ++k) res[k] = fma2(res[k], dup2(a.k_a), dup2(a.k_b));
        }
    } else {
#pragma unroll
        for (int k = 0; k < NB; ++k)
            res[k] = fma2(make_float2(fsqrt(mag2[k].x), fsqrt(mag2[k].y)), dup2(a.k_a), dup2(a.k_b));
    }
    const long long oa = out_row(a, row_a) * (long long)(N / 2);
    const bool has_b = row_a + 1 < a.m;
    const long long ob = has_b ? out_row(a, row_a + 1) * (long long)(N / 2) : 0;
#pragma unroll
    for (int i = 0; i < L::D; ++i)
#pragma unroll
        for (int q = 0; q < L::R / 2; ++q) {
            const int bin = L::bin(t, i, q);
            float2 r = res[i * (L::R / 2) + q];
            if (a.bgv) r = sub2(r, dup2(__ldg(a.bgv + bin)));
            __stcs(a.out + oa + bin, r.x);
            if (has_b) __stcs(a.out + ob + bin, r.y);
        }
}

// One pair's staged rows -> the team's spectrum: the optional bitshift, then
// the packed integer spectrum (8/16-bit samples without rolling-average DC
// removal), rolling-average DC removal (exact sums or the reference's order),
// the exact DC split, or the plain unpack. `smem` is the team's region laid
// out as Layout<N, DT>; returns whether the packed spectrum was written, with
// the split-off DC level in `dc` and the packed taps' bias in `cbias`.
// Ends with the stage consumed but WITHOUT a closing barrier.
template <int N, int DT, class Team>
__device__ __forceinline__ bool pair_unpack(const Team& tm, int t, const ChainArgs& a, unsigned char* smem,
                                            float2& dc, float2& cbias) {
    using LY = Layout<N, DT>;
    using sum_t = typename InTraits<DT>::sum_t;
    constexpr int T = Plan<N>::T;
    float2* spec = reinterpret_cast<float2*>(smem + LY::OFF_SPEC);
    sum_t* pfx = reinterpret_cast<sum_t*>(smem + LY::OFF_PFX);
    sum_t* scan = reinterpret_cast<sum_t*>(smem + LY::OFF_SCAN);
    unsigned char* stages = smem + LY::OFF_STAGE;
    const unsigned char* stage = stages;
    if constexpr (DT == IN_U8 || DT == IN_U16) {
        if (a.bitshift) {
            phase_bitshift<N, DT>(t, stages);
            tm.sync();
        }
    }
    dc = make_float2(0.0f, 0.0f);
    // 8/16-bit samples without rolling-average DC removal: packed integer
    // spectrum (bit-identical taps, half the shared-memory bytes)
    constexpr bool PACKABLE = (DT == IN_U8 || DT == IN_U16);
    const bool packed = PACKABLE && a.dc_window == 0;
    cbias = dup2(8388608.0f);
    if (packed) {
        uint32_t words[16];
        int sa, sb;
        phase_split_load_packed<N, DT>(t, stage, words, &sa, &sb);
        if (a.dc_resp) {
            team_sum2<T, int>(tm, sa, sb, reinterpret_cast<int*>(scan));
            dc = make_float2(split_level((double)sa, N, true), split_level((double)sb, N, true));
            cbias = add2(cbias, dc);  // 2^23 + c, exact for c < 2^23
        }
        phase_store_packed<N>(t, words, reinterpret_cast<uint32_t*>(spec));
    } else if (a.dc_window > 0 && a.dc_ref_order) {
        // Integer samples whose row totals stay below 2^24: every partial sum
        // of the reference's float prefix is an exact integer, so the exact
        // integer prefix gives the same window sums bit for bit (always the
        // case for 8-bit samples, and for 12-bit ones up to N = 4096).
        bool done = false;
        if constexpr (DT != IN_F32) {
            sum_t ta, tb, tot_a, tot_b;
            phase_dc_local<N, DT>(t, stage, &ta, &tb);
            team_exclusive_scan2<T, sum_t>(tm, ta, tb, scan, &tot_a, &tot_b);
            if (dc_prefix_exact_in_float(tot_a) && dc_prefix_exact_in_float(tot_b)) {
                phase_dc_prefix<N, DT>(t, stage, ta, tb, pfx);
                tm.sync();
                phase_dc_apply<N, DT>(t, stage, pfx, a.dc_window, spec);
                done = true;
            } else if constexpr (DT == IN_U16) {
                // the float prefix by segments (phase_dc_refpar_*); the step data
                // live in the spectrum area, which the apply step writes last
                static_assert(RefparArea<N>::BYTES <= LY::SPEC_BYTES, "the step records fit the spectrum area");
                unsigned char* area = smem + LY::OFF_SPEC;
                float* pf = reinterpret_cast<float*>(pfx);
                // each segment's four threads take the exact prefix its owner
                // (thread 4q, the same warp) holds after the scan
                const int ex_a = __shfl_sync(0xffffffffu, (int)ta, (t & 31) & ~3);
                const int ex_b = __shfl_sync(0xffffffffu, (int)tb, (t & 31) & ~3);
                phase_dc_refpar_seg<N>(t, stage, ex_a, ex_b, area);
                tm.sync();
                phase_dc_refpar_walk<N>(t, stage, area);
                tm.sync();
                phase_dc_refpar_fill<N>(t, stage, area, pf);
                tm.sync();
                phase_dc_apply<N, DT, true>(t, stage, pf, a.dc_window, spec);
                done = true;
            }
        }
        if (!done) {
            phase_dc_ref_scan<N, DT>(t, stage, reinterpret_cast<float*>(pfx));
            tm.sync();
            phase_dc_apply<N, DT, true>(t, stage, pfx, a.dc_window, spec);
        }
    } else if (a.dc_window > 0) {
        sum_t ta, tb;
        phase_dc_local<N, DT>(t, stage, &ta, &tb);
        team_exclusive_scan2<T, sum_t>(tm, ta, tb, scan);
        phase_dc_prefix<N, DT>(t, stage, ta, tb, pfx);
        tm.sync();
        phase_dc_apply<N, DT>(t, stage, pfx, a.dc_window, spec);
    } else if (a.dc_resp) {
        using SS = typename SplitSum<DT>::type;
        float2 vals[16];
        SS sa, sb;
        phase_split_load<N, DT>(t, stage, vals, &sa, &sb);
        team_sum2<T, SS>(tm, sa, sb, reinterpret_cast<SS*>(scan));
        dc = make_float2(split_level((double)sa, N, DT != IN_F32), split_level((double)sb, N, DT != IN_F32));
        phase_split_store<N>(t, vals, dc, spec);
    } else {
        phase_unpack<N, DT>(t, stage, spec);
    }
    return packed;
}

// k-linearisation, window and phase of one pair from the team's spectrum
// (the packed integer one when `packed`) into the pass-0 inputs v.
template <int N, int INTERP>
__device__ __forceinline__ void pair_prestage(int t, bool packed, const unsigned char* smem, float2 cbias,
                                              const ChainArgs& a, cp* v) {
    const float2* spec = reinterpret_cast<const float2*>(smem + Layout<N, IN_U16>::OFF_SPEC);
    if (packed) phase_prestage_packed<N, INTERP>(t, reinterpret_cast<const uint32_t*>(spec), cbias, a, v);
    else phase_prestage<N, INTERP>(t, spec, a, v);
}

// The Stockham passes of radix schedule S up to the last one, whose bins stay
// in v (bin layout of LastInfo<N, S>). The exchange buffer aliases the
// spectrum: the first barrier orders every thread's spectrum reads before it.
template <int N, int S, class Team>
__device__ __forceinline__ void pair_fft(const Team& tm, int t, cp* v, const float2* tw, unsigned char* smem) {
    constexpr int NPASS = Plan<N>::NPASS;
    float4* exch = reinterpret_cast<float4*>(smem + Layout<N, IN_U16>::OFF_EXCH);
    fft_twiddle_dft<N, 0, false, S>(t, v, tw);
    tm.sync();  // spec aliases the exchange buffer
    fft_store<N, 0, S>(t, v, exch);
    tm.sync();
    if constexpr (NPASS > 2) {
        fft_load<N>(t, exch, v);
        fft_twiddle_dft<N, 1, false, S>(t, v, tw);
        tm.sync();
        fft_store<N, 1, S>(t, v, exch);
        tm.sync();
    }
    if constexpr (NPASS > 3) {
        fft_load<N>(t, exch, v);
        fft_twiddle_dft<N, 2, false, S>(t, v, tw);
        tm.sync();
        fft_store<N, 2, S>(t, v, exch);
        tm.sync();
    }
    fft_load<N>(t, exch, v);
    fft_twiddle_dft<N, NPASS - 1, false, S>(t, v, tw);
}

// Runs the chain up to the last FFT pass for the pairs p = p0, p0 + step, ...
// (< p_end) whose rows are row0 + 2p and row0 + 2p + 1 (the second one only if
// < row_end), and hands each pair's bins to `sink(t, v, row_a, has_b)`.
// Raw rows are staged by cp.async.bulk into one shared-memory stage: the copy
// of the next pair is issued as soon as this pair's rows are unpacked, so it
// overlaps the resampling, the DFT and the epilogue. Every wait is bounded
// (a.timeout_ns); a timeout sets STATUS_MBAR_TIMEOUT and returns once the copy
// in flight has landed (STATUS_COPY_PENDING if that too runs out).
// `tm` is the team running the pairs (the CTA, or a named-barrier sub-team
// whose shared-memory region starts at smem); S selects the radix schedule.
template <int N, int DT, int INTERP, int S, class Team, class Sink>
__device__ __forceinline__ void run_pairs(const Team& tm, const ChainArgs& a, long long row0, long long row_end,
                                          long long p0, long long p_end, long long step, unsigned char* smem,
                                          Sink& sink) {
    using LY = Layout<N, DT>;
    using raw_t = typename InTraits<DT>::raw_t;

    unsigned char* stages = smem + LY::OFF_STAGE;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + LY::OFF_MBAR);
    int* abort_flag = reinterpret_cast<int*>(smem + LY::OFF_MBAR + 16);

    const int t = tm.tid();
    constexpr uint32_t ROW_BYTES = N * sizeof(raw_t);
    const unsigned char* in = static_cast<const unsigned char*>(a.in);

    if (t == 0) {
        mbar_init(&mbar[0], 1);
        fence_mbar_init();
        *abort_flag = 0;
    }
    tm.sync();

    auto issue = [&](long long pair) {
        const long long r = row0 + 2 * pair;
        const uint32_t rows = (row_end - r) >= 2 ? 2u : 1u;
        const uint32_t bytes = rows * ROW_BYTES;
        fence_proxy_async_smem();
        mbar_expect_tx(&mbar[0], bytes);
        bulk_g2s(stages, in + r * (long long)ROW_BYTES, bytes, &mbar[0]);
    };

    long long item = p0;
    // thread 0: whether a copy was issued for the phase being waited on
    bool issued = false;
    if (t == 0 && item < p_end && !a.debug_skip_first_copy) {
        issue(item);
        issued = true;
    }

    for (int it = 0; item < p_end; item += step, ++it) {
        const long long nxt = item + step;
        const bool ok = (it == 0 && a.debug_abort_first_wait) ? false
                                                               : mbar_wait_bounded(&mbar[0], it & 1, a.timeout_ns);
        if (!ok) *abort_flag = 1;
        tm.sync();
        if (*abort_flag) {
            // A copy issued for this phase may still be writing into this CTA's
            // shared memory and counting against its mbarrier: thread 0 waits it
            // out (a second bound) before the CTA returns, and says so in the
            // status if even that runs out.
            if (t == 0) {
                int st = STATUS_MBAR_TIMEOUT;
                if (issued && !mbar_wait_bounded(&mbar[0], it & 1, a.timeout_ns)) st |= STATUS_COPY_PENDING;
                if (a.status) atomicOr(a.status, st);
            }
            return;
        }
        float2 dc, cbias;
        const bool packed = pair_unpack<N, DT>(tm, t, a, smem, dc, cbias);
        tm.sync();
        if (t == 0) {  // every thread is done with the stage
            issued = nxt < p_end;
            if (issued) issue(nxt);
        }
        cp v[16];
        pair_prestage<N, INTERP>(t, packed, smem, cbias, a, v);
        pair_fft<N, S>(tm, t, v, a.tw, smem);
        const long long ra = row0 + 2 * item;
        sink(t, v, ra, ra + 1 < row_end, dc);
        // the next item's writes to spec/exch come after the barrier at the top
        // of the loop, which every thread reaches only once its sink is done
    }
    tm.sync();  // the caller may reuse the region once the last item's loads are done
}

template <int N, int S, class Team>
struct ImageSink {
    const Team& tm;
    const ChainArgs& a;
    float* scratch;
    __device__ __forceinline__ void operator()(int t, const cp* v, long long row_a, bool has_b, float2 dc) {
        if (a.bins_out) {
            // complex bins after the (optional) FPN subtraction, before magnitude
            using L = LastInfo<N, S>;
#pragma unroll
            for (int i = 0; i < L::D; ++i)
#pragma unroll
                for (int q = 0; q < L::R / 2; ++q) {
                    const int bin = L::bin(t, i, q);
                    cp x = add_dc(a, v[i + q * L::D], bin, dc);
                    if (a.fpn) {
                        const float2 f = __ldg(a.fpn + bin);
                        x.re = sub2(x.re, dup2(f.x));
                        x.im = sub2(x.im, dup2(f.y));
                    }
                    a.bins_out[row_a * (N / 2) + bin] = make_float2(x.re.x, x.im.x);
                    if (has_b) a.bins_out[(row_a + 1) * (N / 2) + bin] = make_float2(x.re.y, x.im.y);
                }
            return;
        }
        epilogue<N, S>(tm, t, v, a, row_a, dc, scratch);
    }
};

// Register cap 128 per thread for every length (8192/N CTAs of N/16 threads
// fill the register file): 16 warps per SM where shared memory allows.
template <int N, int DT, int INTERP>
__global__ void __launch_bounds__(N / 16, 8192 / N) chain_kernel(const ChainArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    using LY = Layout<N, DT>;
    const CtaTeam tm;
    ImageSink<N, 0, CtaTeam> sink{tm, a, reinterpret_cast<float*>(smem + LY::OFF_SCAN)};
    const long long npairs = (a.m + 1) / 2;
    run_pairs<N, DT, INTERP, 0>(tm, a, 0, a.m, blockIdx.x, npairs, gridDim.x, smem, sink);
}

}  // namespace ope_b200

namespace ope_b200 {

// Accumulates, per kept bin, sum re, sum im and sum |z|^2 (double) over the
// A-scans this CTA processes; the minimum-variance mean of
// getMinimumVarianceMean (cpu_kernels.tpp:402-458) is built from these sums.
template <int N>
struct FpnStatsSink {
    using L = LastInfo<N>;
    double acc[L::NB][3];
    __device__ __forceinline__ void reset() {
#pragma unroll
        for (int k = 0; k < L::NB; ++k) acc[k][0] = acc[k][1] = acc[k][2] = 0.0;
    }
    const ChainArgs* args;
    __device__ __forceinline__ void operator()(int t, const cp* v, long long, bool has_b, float2 dc) {
#pragma unroll
        for (int i = 0; i < L::D; ++i)
#pragma unroll
            for (int q = 0; q < L::R / 2; ++q) {
                const cp x = add_dc(*args, v[i + q * L::D], L::bin(t, i, q), dc);
                const int k = i * (L::R / 2) + q;
                double re = x.re.x, im = x.im.x;
                acc[k][0] += re;
                acc[k][1] += im;
                acc[k][2] += re * re + im * im;
                if (has_b) {
                    re = x.re.y;
                    im = x.im.y;
                    acc[k][0] += re;
                    acc[k][1] += im;
                    acc[k][2] += re * re + im * im;
                }
            }
    }
};

// grid = (gx, 8): blockIdx.y is the FPN segment. Segment s covers accumulation
// rows [s*seg_w, (s+1)*seg_w); this buffer holds accumulation rows
// [g0, g0 + rows). Partials: partial[((s*gx + bx)*(N/2) + bin)*3 + k].
template <int N, int DT, int INTERP>
__global__ void __launch_bounds__(N / 16) fpn_stats_kernel(const ChainArgs a, long long g0, long long rows,
                                                             long long seg_w, double* partial) {
    extern __shared__ __align__(128) unsigned char smem[];
    using L = LastInfo<N>;
    const int s = blockIdx.y;
    const long long glo = (long long)s * seg_w, ghi = glo + seg_w;
    long long lo = (glo > g0 ? glo : g0) - g0;
    long long hi = (ghi < g0 + rows ? ghi : g0 + rows) - g0;
    FpnStatsSink<N> sink;
    sink.args = &a;
    sink.reset();
    if (hi > lo) {
        const long long npairs = (hi - lo + 1) / 2;
        run_pairs<N, DT, INTERP, 0>(CtaTeam{}, a, lo, hi, blockIdx.x, npairs, gridDim.x, smem, sink);
    }
    const int t = threadIdx.x;
    double* dst = partial + ((long long)s * gridDim.x + blockIdx.x) * (N / 2) * 3;
#pragma unroll
    for (int i = 0; i < L::D; ++i)
#pragma unroll
        for (int q = 0; q < L::R / 2; ++q) {
            const int bin = L::bin(t, i, q);
            const int k = i * (L::R / 2) + q;
            dst[bin * 3 + 0] = sink.acc[k][0];
            dst[bin * 3 + 1] = sink.acc[k][1];
            dst[bin * 3 + 2] = sink.acc[k][2];
        }
}

}  // namespace ope_b200
