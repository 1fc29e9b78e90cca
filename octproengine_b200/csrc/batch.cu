// Batched chain: many buffers of uneven A-scan length, count, input type,
// resampling mode and window in ONE persistent launch, replayable as a CUDA
// graph, with a per-length autotuner.
//
// No counterpart in the reference, whose backends process one IOBuffer of one
// geometry per call (CpuBackend::Impl::processData, cpu_backend.cpp:169-302;
// CudaBackend::process, cuda_backend.cu:442-773); each buffer here is
// described by an ope_b200_ctx (its ProcessorConfiguration and curves), so
// every buffer gets exactly the chain a single-buffer call would run.
//
// Work decomposition. The buffers are grouped by length N and stage width
// (8/16-bit samples apart from float ones); a group's A-scan pairs are
// numbered consecutively over its buffers. A CTA has 256 threads and, while
// it works on a group, runs 4096/N teams of N/16 threads (each with its own
// named barrier and shared-memory region), every team running the
// single-buffer kernel's pair-of-A-scans pipeline (pair_unpack,
// pair_prestage, pair_fft, the image epilogue) with the input type and
// resampling mode of each pair's buffer chosen at run time. Teams take pairs
// from the group's counter in grabs of `chunk` pairs and stage the next pair
// (of any buffer of the group) while computing the current one, so the
// copy/compute pipeline runs unbroken across grabs and buffers. Each CTA
// starts on the group whose CTA range (proportional to the group's estimated
// work) holds it and then visits the other groups in turn, entering only
// those with pairs left; the last CTA to finish resets the counters, so a
// captured graph replays without a memset.
// The autotuner picks the grab size and the FFT radix schedule per length by
// timing this batch's own buffers of that length.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/ope_b200.h"
#include "chain_device.cuh"
#include "tables.h"

namespace ope_b200 {

int ctx_batch_args(ope_b200_ctx* c, ChainArgs* a, int* n, int* in_kind, int* interp, int* device);
const char* ctx_error(const ope_b200_ctx* c);

constexpr int BATCH_THREADS = 256;
constexpr int BATCH_MAX_GROUPS = 6;  // one per supported length and stage width

struct BatchDesc {
    ChainArgs a;
    int n, in_kind, interp, group;
    long long pair0;   // first pair of this buffer in its group's numbering
    long long npairs;  // (m + 1) / 2
};

struct GroupDesc {
    int n, sched;
    int first;          // index of the group's first descriptor (its buffers are consecutive)
    int count;
    long long npairs;   // pairs of all the group's buffers
    int chunk;          // pairs per grab
    int cta_begin;      // first CTA that starts on this group
    int wide;           // 1: float samples (4-byte stage), 0: 8/16-bit samples (2-byte stage)
    int pad;
};

// One team's region: the spectrum, prefix, scan and exchange areas and the
// stage at the offsets of Layout<N, DT> (the same for 8-, 16-bit and float
// samples, so pair_unpack<N, DT> of any of them works in it), the stage sized
// for W-byte samples (W = 2 for a group of 8/16-bit buffers, 4 for float
// ones), then the control words. Groups are split by stage width so that a
// group of 8/16-bit buffers keeps the single-buffer kernel's shared-memory
// footprint, which leaves the L1 share of the SM's memory to the table reads.
template <int N, int W>
struct BatchRegion {
    using LY = Layout<N, IN_U16>;
    static_assert(Layout<N, IN_U8>::OFF_STAGE == LY::OFF_STAGE && Layout<N, IN_F32>::OFF_STAGE == LY::OFF_STAGE &&
                      Layout<N, IN_U8>::OFF_SCAN == LY::OFF_SCAN && Layout<N, IN_F32>::OFF_SCAN == LY::OFF_SCAN &&
                      Layout<N, IN_U8>::OFF_PFX == LY::OFF_PFX && Layout<N, IN_F32>::OFF_PFX == LY::OFF_PFX,
                  "batched teams share one layout for every input type");
    static constexpr int TEAMS = BATCH_THREADS / (N / 16);
    static constexpr int CTL = LY::OFF_STAGE + 2 * N * W;  // control words after the stage
    static constexpr int BYTES = (CTL + 64 + 127) / 128 * 128;
};

// A team's control words (64 bytes at BatchRegion::CTL): its mbarrier, the
// abort flag, the staged pair (descriptor, pair within its buffer) and
// thread 0's grab [lo, hi) and descriptor cursor.
struct TeamCtl {
    uint64_t mbar;
    int pad0, pad1;
    int abort;
    int next_desc;  // -1: no further pair
    long long next_pair;
    long long grab_lo, grab_hi;
    int cursor;
    int pad2;
};
static_assert(sizeof(TeamCtl) <= 64, "team control words fit their 64-byte slot");

__device__ __forceinline__ uint32_t in_bytes(int kind) { return kind == IN_U8 ? 1u : kind == IN_U16 ? 2u : 4u; }

// Thread 0 of a team: takes the team's next pair of group g (a new grab of
// g.chunk pairs from `counter` when the current one is used up), publishes it
// in the control words and issues the copy of its rows into the stage; or
// publishes "none". A team's pairs only increase, so the descriptor cursor
// only moves forward.
template <int N, int W>
__device__ __forceinline__ void team_stage_next(const BatchDesc* __restrict__ descs, const GroupDesc* g,
                                                unsigned long long* counter, unsigned char* my) {
    using R = BatchRegion<N, W>;
    using LY = typename R::LY;
    TeamCtl* c = reinterpret_cast<TeamCtl*>(my + R::CTL);
    if (c->grab_lo >= c->grab_hi) {
        const long long s = (long long)atomicAdd(counter, (unsigned long long)g->chunk);
        if (s >= g->npairs) {
            c->next_desc = -1;
            return;
        }
        c->grab_lo = s;
        c->grab_hi = (s + g->chunk < g->npairs) ? s + g->chunk : g->npairs;
    }
    const long long p = c->grab_lo++;
    int di = c->cursor;
    while (descs[di].pair0 + descs[di].npairs <= p) ++di;
    c->cursor = di;
    const BatchDesc& D = descs[di];
    const long long lp = p - D.pair0;
    const long long r = 2 * lp;
    const uint32_t row_bytes = (uint32_t)N * in_bytes(D.in_kind);
    const uint32_t bytes = ((D.a.m - r) >= 2 ? 2u : 1u) * row_bytes;
    c->next_desc = di;
    c->next_pair = lp;
    fence_proxy_async_smem();
    mbar_expect_tx(&c->mbar, bytes);
    bulk_g2s(my + LY::OFF_STAGE, static_cast<const unsigned char*>(D.a.in) + r * (long long)row_bytes, bytes,
             &c->mbar);
}

// One team's share of group g: the pairs team_stage_next hands it, one at a
// time through the pipeline, the next pair's copy issued as soon as the
// current pair's rows are unpacked. Returns whether a bounded wait ran out
// (the team stops; the status word says so).
template <int N, int S, int W>
__device__ __forceinline__ bool group_run(const BatchDesc* __restrict__ descs, const GroupDesc* g,
                                          unsigned long long* counter, unsigned char* smem) {
    using R = BatchRegion<N, W>;
    using LY = typename R::LY;
    constexpr int T = N / 16;
    const int team = threadIdx.x / T;
    const SubTeam tm{team * T, 1 + team, T};
    unsigned char* my = smem + team * R::BYTES;
    TeamCtl* ctl = reinterpret_cast<TeamCtl*>(my + R::CTL);
    const int t = tm.tid();
    if (t == 0) {
        mbar_init(&ctl->mbar, 1);
        fence_mbar_init();
        ctl->abort = 0;
        ctl->grab_lo = ctl->grab_hi = 0;
        ctl->cursor = g->first;
        team_stage_next<N, W>(descs, g, counter, my);
    }
    tm.sync();
    for (int it = 0;; ++it) {
        const int cd = ctl->next_desc;
        if (cd < 0) break;
        const long long lp = ctl->next_pair;
        const ChainArgs& a = descs[cd].a;
        const bool ok = mbar_wait_bounded(&ctl->mbar, it & 1, a.timeout_ns);
        if (!ok) ctl->abort = 1;
        tm.sync();
        if (ctl->abort) {
            // as run_pairs: wait out the copy of this phase (a second bound) before leaving
            if (t == 0) {
                int st = STATUS_MBAR_TIMEOUT;
                if (!mbar_wait_bounded(&ctl->mbar, it & 1, a.timeout_ns)) st |= STATUS_COPY_PENDING;
                if (a.status) atomicOr(a.status, st);
            }
            break;
        }
        float2 dc, cbias;
        bool packed;
        const int kind = descs[cd].in_kind;
        if constexpr (W == 4) {
            (void)kind;
            packed = pair_unpack<N, IN_F32>(tm, t, a, my, dc, cbias);
        } else {
            if (kind == IN_U8) packed = pair_unpack<N, IN_U8>(tm, t, a, my, dc, cbias);
            else packed = pair_unpack<N, IN_U16>(tm, t, a, my, dc, cbias);
        }
        tm.sync();
        // every thread is done with the stage and has read next_*
        if (t == 0) team_stage_next<N, W>(descs, g, counter, my);
        cp v[16];
        const int interp = descs[cd].interp;
        if (interp == INTERP_CUBIC) pair_prestage<N, INTERP_CUBIC>(t, packed, my, cbias, a, v);
        else if (interp == INTERP_LINEAR) pair_prestage<N, INTERP_LINEAR>(t, packed, my, cbias, a, v);
        else if (interp == INTERP_LANCZOS) pair_prestage<N, INTERP_LANCZOS>(t, packed, my, cbias, a, v);
        else pair_prestage<N, INTERP_NONE>(t, packed, my, cbias, a, v);
        pair_fft<N, S>(tm, t, v, a.tw, my);
        ImageSink<N, S, SubTeam> sink{tm, a, reinterpret_cast<float*>(my + LY::OFF_SCAN)};
        const long long ra = 2 * lp;
        sink(t, v, ra, ra + 1 < a.m, dc);
    }
    tm.sync();
    const bool aborted = ctl->abort != 0;
    // the region may hold another length's layout next (an aborted team's
    // copy may still be pending: its CTA takes no further group)
    if (t == 0 && !aborted) mbar_inval(&ctl->mbar);
    return aborted;
}

template <int W>
__device__ __forceinline__ bool group_dispatch(const BatchDesc* __restrict__ descs, const GroupDesc& g,
                                               unsigned long long* counter, unsigned char* smem) {
    switch (g.n) {
        case 1024:
            if (g.sched == 0) return group_run<1024, 0, W>(descs, &g, counter, smem);
            if (g.sched == 1) return group_run<1024, 1, W>(descs, &g, counter, smem);
            return group_run<1024, 2, W>(descs, &g, counter, smem);
        case 2048:
            if (g.sched == 0) return group_run<2048, 0, W>(descs, &g, counter, smem);
            if (g.sched == 1) return group_run<2048, 1, W>(descs, &g, counter, smem);
            return group_run<2048, 2, W>(descs, &g, counter, smem);
        default: return group_run<4096, 0, W>(descs, &g, counter, smem);
    }
}

__global__ void __launch_bounds__(BATCH_THREADS, 2)
    batch_kernel(const BatchDesc* __restrict__ descs, const GroupDesc* __restrict__ groups, int ngroups,
                 unsigned long long* counters) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int enter, aborted;
    int g0 = 0;
    for (int g = 1; g < ngroups; ++g)
        if (groups[g].cta_begin <= (int)blockIdx.x) g0 = g;
    if (threadIdx.x == 0) aborted = 0;
    for (int k = 0; k < ngroups; ++k) {
        const int gi = (g0 + k) % ngroups;
        const GroupDesc& g = groups[gi];
        if (threadIdx.x == 0)
            enter = !aborted &&
                    *reinterpret_cast<volatile unsigned long long*>(counters + gi) < (unsigned long long)g.npairs;
        __syncthreads();
        if (enter) {
            bool ab;
            if (g.wide) ab = group_dispatch<4>(descs, g, counters + gi, smem);
            else ab = group_dispatch<2>(descs, g, counters + gi, smem);
            if (ab) aborted = 1;  // benign race: every writer stores 1
        }
        __syncthreads();  // every team is done before shared memory takes another group's layout
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(counters + ngroups, 1ull) == (unsigned long long)gridDim.x - 1) {
            // every CTA has left the loop: nobody reads the counters any more
            for (int g = 0; g <= ngroups; ++g) counters[g] = 0;
            __threadfence();
        }
    }
}

template <int W>
int host_region_w(int n) {
    return n == 1024 ? BatchRegion<1024, W>::BYTES : n == 2048 ? BatchRegion<2048, W>::BYTES : BatchRegion<4096, W>::BYTES;
}
int host_region(int n, bool wide) { return wide ? host_region_w<4>(n) : host_region_w<2>(n); }
int host_teams(int n) { return BATCH_THREADS / (n / 16); }

// Relative cost of one pair, for the CTAs' starting groups only (the groups'
// counters balance the rest): N log N, Lanczos-8 resampling about 1.8x.
double pair_cost(int n, int interp) {
    int lg = 0;
    while ((1 << lg) < n) ++lg;
    return (double)n * lg * (interp == INTERP_LANCZOS ? 1.8 : 1.0);
}

// Radix plans per length: 1024 = 16*16*4, 4*16*16, 16*4*16; 2048 = 16*16*8,
// 8*16*16, 16*8*16; 4096 = 16*16*16 (one plan).
int num_schedules(int n) { return (n == 1024 || n == 2048) ? 3 : 1; }

}  // namespace ope_b200

using namespace ope_b200;

struct ope_b200_batch {
    int device = 0;
    std::vector<ope_b200_batch_item> items;
    std::vector<BatchDesc> base;  // per item, before tuning
    std::map<int, std::pair<int, int>> tuning;  // n -> (pairs per grab, schedule)
    std::map<int, float> tuned_us;
    std::map<std::pair<int, int>, float2*> tw;  // (n, schedule) -> twiddles
    unsigned char* d_block = nullptr;  // plain launches: descriptors, then group descriptors
    size_t d_cap = 0;
    unsigned char* g_block = nullptr;  // the captured graph's own copy
    size_t g_cap = 0;
    cudaEvent_t last_launch = nullptr;
    unsigned long long* d_counter = nullptr;  // one per group, then the CTAs-done count
    int sms = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap_stream = nullptr;
    std::string err;
};

namespace {

int bfail(ope_b200_batch* b, int code, const std::string& m) {
    if (b) b->err = m;
    return code;
}

#define BATCH_CU(b, call)                                                                              \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return bfail(b, OPE_B200_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void drop_graph(ope_b200_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

constexpr int kDefaultChunk = 2;

struct LaunchPlan {
    const BatchDesc* descs = nullptr;
    const GroupDesc* groups = nullptr;
    int ngroups = 0, smem = 0, grid = 0;
};

// Descriptors and group descriptors of the items selected by `pick` under the
// current tuning, uploaded to `*dst` (grown as needed) with a synchronous
// copy, and the launch configuration they need.
int prepare(ope_b200_batch* b, const std::vector<int>& pick, unsigned char** dst, size_t* cap, LaunchPlan* lp) {
    // groups: one per (length, stage width), float buffers apart from 8/16-bit ones
    std::map<std::pair<int, int>, std::vector<int>> by_n;
    for (int i : pick) by_n[{b->base[i].n, b->base[i].in_kind == IN_F32 ? 1 : 0}].push_back(i);
    std::vector<BatchDesc> v;
    std::vector<GroupDesc> gs;
    std::vector<double> cost;
    double total = 0.0;
    int sm = 0;
    long long team_rounds = 0;  // pairs / teams per CTA, summed over groups
    for (const auto& kv : by_n) {
        const int n = kv.first.first;
        const auto tn = b->tuning.count(n) ? b->tuning[n] : std::make_pair(kDefaultChunk, 0);
        GroupDesc g{};
        g.n = n;
        g.wide = kv.first.second;
        g.sched = tn.second < num_schedules(n) ? tn.second : 0;
        g.chunk = tn.first;
        g.first = (int)v.size();
        g.count = (int)kv.second.size();
        long long p = 0;
        double c = 0.0;
        for (int i : kv.second) {
            BatchDesc d = b->base[i];
            d.a.tw = b->tw[{n, g.sched}];
            d.group = (int)gs.size();
            d.pair0 = p;
            d.npairs = (d.a.m + 1) / 2;
            p += d.npairs;
            c += (double)d.npairs * pair_cost(n, d.interp);
            v.push_back(d);
        }
        g.npairs = p;
        gs.push_back(g);
        cost.push_back(c);
        total += c;
        sm = std::max(sm, host_teams(n) * host_region(n, g.wide != 0));
        team_rounds += (p + host_teams(n) - 1) / host_teams(n);
    }
    const size_t bytes = v.size() * sizeof(BatchDesc) + gs.size() * sizeof(GroupDesc);
    if (bytes > *cap) {
        cudaFree(*dst);
        *dst = nullptr;
        BATCH_CU(b, cudaMalloc(dst, bytes));
        *cap = bytes;
    }
    BATCH_CU(b, cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    int occ = 0;
    BATCH_CU(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, BATCH_THREADS, sm));
    if (occ < 1) return bfail(b, OPE_B200_E_UNSUPPORTED, "batch kernel does not fit on an SM");
    long long grid = (long long)occ * b->sms;
    if (grid > team_rounds) grid = team_rounds;
    if (grid < 1) grid = 1;
    double cum = 0.0;
    for (size_t k = 0; k < gs.size(); ++k) {
        gs[k].cta_begin = (int)(grid * cum / total + 0.5);
        cum += cost[k];
    }
    std::vector<unsigned char> host(bytes);
    std::memcpy(host.data(), v.data(), v.size() * sizeof(BatchDesc));
    std::memcpy(host.data() + v.size() * sizeof(BatchDesc), gs.data(), gs.size() * sizeof(GroupDesc));
    BATCH_CU(b, cudaMemcpy(*dst, host.data(), bytes, cudaMemcpyHostToDevice));
    lp->descs = reinterpret_cast<const BatchDesc*>(*dst);
    lp->groups = reinterpret_cast<const GroupDesc*>(*dst + v.size() * sizeof(BatchDesc));
    lp->ngroups = (int)gs.size();
    lp->smem = sm;
    lp->grid = (int)grid;
    return OPE_B200_OK;
}

int enqueue(ope_b200_batch* b, const LaunchPlan& lp, cudaStream_t s) {
    batch_kernel<<<(unsigned)lp.grid, BATCH_THREADS, lp.smem, s>>>(lp.descs, lp.groups, lp.ngroups, b->d_counter);
    BATCH_CU(b, cudaGetLastError());
    return OPE_B200_OK;
}

// Plain launch: the descriptor upload is synchronous, so wait for the
// previous launch of this batch (which may still read the descriptors).
int launch(ope_b200_batch* b, const std::vector<int>& pick, cudaStream_t s) {
    if (b->last_launch) BATCH_CU(b, cudaEventSynchronize(b->last_launch));
    LaunchPlan lp;
    int rc = prepare(b, pick, &b->d_block, &b->d_cap, &lp);
    if (rc != OPE_B200_OK) return rc;
    rc = enqueue(b, lp, s);
    if (rc != OPE_B200_OK) return rc;
    BATCH_CU(b, cudaEventRecord(b->last_launch, s));
    return OPE_B200_OK;
}

std::vector<int> all_items(const ope_b200_batch* b) {
    std::vector<int> v(b->items.size());
    for (size_t i = 0; i < v.size(); ++i) v[i] = (int)i;
    return v;
}

}  // namespace

extern "C" {

int ope_b200_batch_create(const ope_b200_batch_item* items, int32_t count, ope_b200_batch** out) {
    if (!out || !items || count < 1) return OPE_B200_E_INVALID;
    *out = nullptr;
    auto* b = new ope_b200_batch();
    auto bail = [&](int rc) {
        ope_b200_batch_destroy(b);
        return rc;
    };
    for (int i = 0; i < count; ++i) {
        const ope_b200_batch_item& it = items[i];
        if (!it.ctx || !it.d_in || !it.d_out || it.num_ascans < 1) return bail(OPE_B200_E_INVALID);
        if ((reinterpret_cast<uintptr_t>(it.d_in) & 15u) != 0 || (reinterpret_cast<uintptr_t>(it.d_out) & 3u) != 0)
            return bail(OPE_B200_E_INVALID);
        BatchDesc d{};
        int dev = 0;
        int rc = ctx_batch_args(it.ctx, &d.a, &d.n, &d.in_kind, &d.interp, &dev);
        if (rc != OPE_B200_OK) return bail(rc);
        if (d.n != 1024 && d.n != 2048 && d.n != 4096) return bail(OPE_B200_E_UNSUPPORTED);
        if (d.in_kind != IN_U8 && d.in_kind != IN_U16 && d.in_kind != IN_F32) return bail(OPE_B200_E_UNSUPPORTED);
        if (i == 0) b->device = dev;
        if (dev != b->device) return bail(OPE_B200_E_INVALID);
        d.a.in = it.d_in;
        d.a.out = it.d_out;
        d.a.m = it.num_ascans;
        d.a.bscans = static_cast<int>((it.num_ascans + d.a.ascans_per_bscan - 1) / d.a.ascans_per_bscan);
        b->items.push_back(it);
        b->base.push_back(d);
    }
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, (BATCH_MAX_GROUPS + 1) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(b->d_counter, 0, (BATCH_MAX_GROUPS + 1) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->last_launch, cudaEventDisableTiming);
    for (const BatchDesc& d : b->base)
        for (int s = 0; s < num_schedules(d.n) && e == cudaSuccess; ++s) {
            if (b->tw.count({d.n, s})) continue;
            const std::vector<float2> t = build_twiddles(d.n, s);
            float2* p = nullptr;
            e = cudaMalloc(&p, t.size() * sizeof(float2));
            if (e == cudaSuccess) {
                b->tw[{d.n, s}] = p;
                e = cudaMemcpy(p, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice);
            }
        }
    if (e != cudaSuccess) return bail(OPE_B200_E_CUDA);
    *out = b;
    return OPE_B200_OK;
}

void ope_b200_batch_destroy(ope_b200_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    drop_graph(b);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    if (b->last_launch) cudaEventDestroy(b->last_launch);
    for (auto& kv : b->tw) cudaFree(kv.second);
    cudaFree(b->d_block);
    cudaFree(b->g_block);
    cudaFree(b->d_counter);
    delete b;
}

const char* ope_b200_batch_last_error(const ope_b200_batch* b) { return b ? b->err.c_str() : "null batch"; }

int ope_b200_batch_set_tuning(ope_b200_batch* b, int32_t n, int32_t pairs_per_team, int32_t radix_schedule) {
    if (!b) return OPE_B200_E_INVALID;
    if (pairs_per_team < 1 || pairs_per_team > 1024 || radix_schedule < 0)
        return bfail(b, OPE_B200_E_INVALID, "pairs_per_team must be in [1, 1024] and radix_schedule >= 0");
    if (radix_schedule >= num_schedules(n))
        return bfail(b, OPE_B200_E_INVALID, "radix_schedule out of range for this length (0..2 at 1024 and 2048, "
                                             "0 at 4096)");
    b->tuning[n] = {pairs_per_team, radix_schedule};
    drop_graph(b);
    return OPE_B200_OK;
}

int ope_b200_batch_get_tuning(ope_b200_batch* b, int32_t n, int32_t* pairs_per_team, int32_t* radix_schedule,
                              float* best_us) {
    if (!b) return OPE_B200_E_INVALID;
    const auto tn = b->tuning.count(n) ? b->tuning[n] : std::make_pair(kDefaultChunk, 0);
    if (pairs_per_team) *pairs_per_team = tn.first;
    if (radix_schedule) *radix_schedule = tn.second;
    if (best_us) *best_us = b->tuned_us.count(n) ? b->tuned_us[n] : -1.0f;
    return OPE_B200_OK;
}

int ope_b200_batch_run(ope_b200_batch* b, void* stream) {
    if (!b) return OPE_B200_E_INVALID;
    BATCH_CU(b, cudaSetDevice(b->device));
    return launch(b, all_items(b), static_cast<cudaStream_t>(stream));
}

int ope_b200_batch_run_graph(ope_b200_batch* b, void* stream) {
    if (!b) return OPE_B200_E_INVALID;
    BATCH_CU(b, cudaSetDevice(b->device));
    if (!b->exec) {
        // the graph gets its own descriptor copy, uploaded before the capture;
        // only the kernel launch is captured
        BATCH_CU(b, cudaDeviceSynchronize());
        LaunchPlan lp;
        int rc = prepare(b, all_items(b), &b->g_block, &b->g_cap, &lp);
        if (rc != OPE_B200_OK) return rc;
        BATCH_CU(b, cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue(b, lp, b->cap_stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
        if (rc != OPE_B200_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        BATCH_CU(b, e);
        b->graph = g;
        BATCH_CU(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    BATCH_CU(b, cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)));
    return OPE_B200_OK;
}

int ope_b200_batch_autotune(ope_b200_batch* b, int32_t reps) {
    if (!b) return OPE_B200_E_INVALID;
    if (reps < 1) reps = 3;
    BATCH_CU(b, cudaSetDevice(b->device));
    cudaStream_t s = b->cap_stream;
    cudaEvent_t e0, e1;
    BATCH_CU(b, cudaEventCreate(&e0));
    BATCH_CU(b, cudaEventCreate(&e1));
    std::map<int, std::vector<int>> by_len;
    for (size_t i = 0; i < b->base.size(); ++i) by_len[b->base[i].n].push_back((int)i);
    static const int kPairs[] = {1, 2, 4, 8};
    int rc = OPE_B200_OK;
    for (auto& kv : by_len) {
        const int n = kv.first;
        float best = 1e30f;
        std::pair<int, int> best_cfg{kDefaultChunk, 0};
        for (int sched = 0; sched < num_schedules(n) && rc == OPE_B200_OK; ++sched)
            for (int pp : kPairs) {
                b->tuning[n] = {pp, sched};
                rc = launch(b, kv.second, s);  // warm-up
                for (int r = 0; r < reps && rc == OPE_B200_OK; ++r) {
                    cudaEventRecord(e0, s);
                    rc = launch(b, kv.second, s);
                    cudaEventRecord(e1, s);
                    cudaEventSynchronize(e1);
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (ms * 1000.0f < best) {
                        best = ms * 1000.0f;
                        best_cfg = {pp, sched};
                    }
                }
                if (rc != OPE_B200_OK) break;
            }
        b->tuning[n] = best_cfg;
        b->tuned_us[n] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graph(b);
    if (rc == OPE_B200_OK) BATCH_CU(b, cudaStreamSynchronize(s));
    return rc;
}

}  // extern "C"
