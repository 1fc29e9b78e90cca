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
// Work decomposition. A CTA has 256 threads; a buffer of N samples per A-scan
// is processed by teams of N/16 threads (4096/N teams per CTA, each with its
// own named barrier and shared-memory region), every team running the same
// pair-of-A-scans pipeline as the single-buffer kernel (run_pairs). The
// buffers' A-scan pairs are cut into units of teams x pairs_per_team pairs;
// persistent CTAs take units from a global counter (the last CTA to finish
// resets it, so a captured graph replays without a memset). The autotuner
// picks pairs_per_team (the A-scans each CTA takes per grab) and the FFT radix
// schedule per length by timing this batch's own buffers of that length.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
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

struct BatchDesc {
    ChainArgs a;
    int n, in_kind, interp, sched;
    int teams;           // teams of n/16 threads per CTA
    int pairs_per_team;  // pairs each team takes per unit
    int region;          // bytes of shared memory per team
    int pad;
    long long unit0, units;  // this buffer's units in the global numbering
};

template <int N, int DT>
constexpr int team_region() {
    return ((Layout<N, DT>::TOTAL + 127) / 128) * 128;
}

template <int N, int DT, int INTERP, int S>
__device__ __noinline__ void batch_team_run(const BatchDesc& d, long long u, unsigned char* smem) {
    constexpr int T = N / 16;
    const int team = threadIdx.x / T;
    if (team >= d.teams) return;
    const SubTeam tm{team * T, 1 + team, T};
    unsigned char* my = smem + team * d.region;
    const long long npairs = (d.a.m + 1) / 2;
    const long long per_unit = (long long)d.pairs_per_team * d.teams;
    const long long p0 = (u - d.unit0) * per_unit;
    const long long p_end = (p0 + per_unit < npairs) ? p0 + per_unit : npairs;
    ImageSink<N, S, SubTeam> sink{tm, d.a, reinterpret_cast<float*>(my + Layout<N, DT>::OFF_SCAN)};
    run_pairs<N, DT, INTERP, S>(tm, d.a, 0, d.a.m, p0 + team, p_end, d.teams, my, sink);
    tm.sync();
    if (tm.tid() == 0) {  // the region may hold another layout in the next unit
        uint64_t* mbar = reinterpret_cast<uint64_t*>(my + Layout<N, DT>::OFF_MBAR);
        mbar_inval(&mbar[0]);
    }
}

template <int N, int S>
__device__ __forceinline__ void dispatch_dt_interp(const BatchDesc& d, long long u, unsigned char* smem) {
#define OPE_B200_BATCH_INTERP(DT)                                                              \
    switch (d.interp) {                                                                        \
        case INTERP_NONE: batch_team_run<N, DT, INTERP_NONE, S>(d, u, smem); break;            \
        case INTERP_LINEAR: batch_team_run<N, DT, INTERP_LINEAR, S>(d, u, smem); break;        \
        case INTERP_CUBIC: batch_team_run<N, DT, INTERP_CUBIC, S>(d, u, smem); break;          \
        default: batch_team_run<N, DT, INTERP_LANCZOS, S>(d, u, smem); break;                  \
    }
    switch (d.in_kind) {
        case IN_U8: OPE_B200_BATCH_INTERP(IN_U8) break;
        case IN_U16: OPE_B200_BATCH_INTERP(IN_U16) break;
        default: OPE_B200_BATCH_INTERP(IN_F32) break;
    }
#undef OPE_B200_BATCH_INTERP
}

__global__ void __launch_bounds__(BATCH_THREADS, 2)
    batch_kernel(const BatchDesc* __restrict__ descs, int ndesc, long long total_units, unsigned long long* counter) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(16) BatchDesc sd;
    __shared__ long long su;
    __shared__ int sb;
    for (;;) {
        if (threadIdx.x == 0) {
            su = (long long)atomicAdd(counter, 1ull);
            int b = 0;
            if (su < total_units)
                while (b + 1 < ndesc && descs[b + 1].unit0 <= su) ++b;
            sb = b;
        }
        __syncthreads();
        const long long u = su;
        if (u >= total_units) break;
        {
            const int* src = reinterpret_cast<const int*>(descs + sb);
            int* dst = reinterpret_cast<int*>(&sd);
            for (int k = threadIdx.x; k < (int)(sizeof(BatchDesc) / 4); k += BATCH_THREADS) dst[k] = src[k];
        }
        __syncthreads();
        switch (sd.n) {
            case 1024:
                if (sd.sched == 0) dispatch_dt_interp<1024, 0>(sd, u, smem);
                else if (sd.sched == 1) dispatch_dt_interp<1024, 1>(sd, u, smem);
                else dispatch_dt_interp<1024, 2>(sd, u, smem);
                break;
            case 2048:
                if (sd.sched == 0) dispatch_dt_interp<2048, 0>(sd, u, smem);
                else if (sd.sched == 1) dispatch_dt_interp<2048, 1>(sd, u, smem);
                else dispatch_dt_interp<2048, 2>(sd, u, smem);
                break;
            default: dispatch_dt_interp<4096, 0>(sd, u, smem); break;
        }
        __syncthreads();  // every team is done before the next unit re-lays out shared memory
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(counter + 1, 1ull) == (unsigned long long)gridDim.x - 1) {
            counter[0] = 0;  // every CTA has left the loop: nobody reads the counter any more
            counter[1] = 0;
            __threadfence();
        }
    }
}

int host_team_region(int n, int kind) {
    switch (n) {
        case 1024: return kind == IN_U8 ? team_region<1024, IN_U8>() : kind == IN_U16 ? team_region<1024, IN_U16>()
                                                                                       : team_region<1024, IN_F32>();
        case 2048: return kind == IN_U8 ? team_region<2048, IN_U8>() : kind == IN_U16 ? team_region<2048, IN_U16>()
                                                                                       : team_region<2048, IN_F32>();
        case 4096: return kind == IN_U8 ? team_region<4096, IN_U8>() : kind == IN_U16 ? team_region<4096, IN_U16>()
                                                                                       : team_region<4096, IN_F32>();
        default: return 0;
    }
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
    std::map<int, std::pair<int, int>> tuning;  // n -> (pairs_per_team, schedule)
    std::map<int, float> tuned_us;
    std::map<std::pair<int, int>, float2*> tw;  // (n, schedule) -> twiddles
    BatchDesc* d_descs = nullptr;  // plain launches
    int d_cap = 0;
    BatchDesc* g_descs = nullptr;  // the captured graph's own copy
    int g_cap = 0;
    cudaEvent_t last_launch = nullptr;
    unsigned long long* d_counter = nullptr;
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

struct LaunchPlan {
    long long units = 0;
    int smem = 0, ndesc = 0, grid = 0;
};

// Descriptors of the items selected by `pick` under the current tuning,
// uploaded to `dst` (grown as needed) with a synchronous copy, and the launch
// configuration they need.
int prepare(ope_b200_batch* b, const std::vector<int>& pick, BatchDesc** dst, int* cap, LaunchPlan* lp) {
    std::vector<BatchDesc> v;
    long long u = 0;
    int sm = 0;
    for (int i : pick) {
        BatchDesc d = b->base[i];
        const auto tn = b->tuning.count(d.n) ? b->tuning[d.n] : std::make_pair(4, 0);
        d.pairs_per_team = tn.first;
        d.sched = tn.second < num_schedules(d.n) ? tn.second : 0;
        d.a.tw = b->tw[{d.n, d.sched}];
        const long long npairs = (d.a.m + 1) / 2;
        const long long per_unit = (long long)d.pairs_per_team * d.teams;
        d.unit0 = u;
        d.units = (npairs + per_unit - 1) / per_unit;
        u += d.units;
        sm = std::max(sm, d.teams * d.region);
        v.push_back(d);
    }
    if ((int)v.size() > *cap) {
        cudaFree(*dst);
        *dst = nullptr;
        BATCH_CU(b, cudaMalloc(dst, v.size() * sizeof(BatchDesc)));
        *cap = (int)v.size();
    }
    BATCH_CU(b, cudaMemcpy(*dst, v.data(), v.size() * sizeof(BatchDesc), cudaMemcpyHostToDevice));
    BATCH_CU(b, cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    int occ = 0;
    BATCH_CU(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, BATCH_THREADS, sm));
    if (occ < 1) return bfail(b, OPE_B200_E_UNSUPPORTED, "batch kernel does not fit on an SM");
    long long grid = (long long)occ * b->sms;
    if (grid > u) grid = u;
    if (grid < 1) grid = 1;
    lp->units = u;
    lp->smem = sm;
    lp->ndesc = (int)v.size();
    lp->grid = (int)grid;
    return OPE_B200_OK;
}

int enqueue(ope_b200_batch* b, const BatchDesc* descs, const LaunchPlan& lp, cudaStream_t s) {
    batch_kernel<<<(unsigned)lp.grid, BATCH_THREADS, lp.smem, s>>>(descs, lp.ndesc, lp.units, b->d_counter);
    BATCH_CU(b, cudaGetLastError());
    return OPE_B200_OK;
}

// Plain launch: the descriptor upload is synchronous, so wait for the
// previous launch of this batch (which may still read the descriptors).
int launch(ope_b200_batch* b, const std::vector<int>& pick, cudaStream_t s) {
    if (b->last_launch) BATCH_CU(b, cudaEventSynchronize(b->last_launch));
    LaunchPlan lp;
    int rc = prepare(b, pick, &b->d_descs, &b->d_cap, &lp);
    if (rc != OPE_B200_OK) return rc;
    rc = enqueue(b, b->d_descs, lp, s);
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
        d.teams = BATCH_THREADS / (d.n / 16);
        d.region = host_team_region(d.n, d.in_kind);
        b->items.push_back(it);
        b->base.push_back(d);
    }
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(b->d_counter, 0, 2 * sizeof(unsigned long long));
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
    cudaFree(b->d_descs);
    cudaFree(b->g_descs);
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
    const auto tn = b->tuning.count(n) ? b->tuning[n] : std::make_pair(4, 0);
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
        int rc = prepare(b, all_items(b), &b->g_descs, &b->g_cap, &lp);
        if (rc != OPE_B200_OK) return rc;
        BATCH_CU(b, cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue(b, b->g_descs, lp, b->cap_stream);
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
    static const int kPairs[] = {1, 2, 4, 8, 16, 32};
    int rc = OPE_B200_OK;
    for (auto& kv : by_len) {
        const int n = kv.first;
        float best = 1e30f;
        std::pair<int, int> best_cfg{4, 0};
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
