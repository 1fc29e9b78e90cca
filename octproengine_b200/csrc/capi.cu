// C ABI of the B200 chain backend: context, curve tables, launches.
//
// Replaces the per-frame work of the reference ProcessingBackend
// implementations (CpuBackend::Impl::processData, cpu_backend.cpp:169-302;
// CudaBackend::process, cuda_backend.cu:442-773) with one fused kernel launch
// per buffer. Host tables derived from the curves are double-buffered on the
// device: a curve update fills the slot no in-flight launch reads (waiting on
// that slot's last-use event) and then switches to it, so hot-swaps are
// ordered against frames already enqueued (the reference CUDA backend is not,
// cuda_backend.cu:784-828).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ope_b200.h"
#include "chain_launch.h"
#include "fpn.h"
#include "postproc.h"
#include "tables.h"

using namespace ope_b200;

namespace {

// ope::DataType values (include/types.h:6-19)
enum : int {
    DT_UINT8 = 1, DT_UINT16 = 2, DT_UINT32 = 3, DT_UINT64 = 4, DT_INT8 = 5, DT_INT16 = 6,
    DT_INT32 = 7, DT_INT64 = 8, DT_FLOAT32 = 9, DT_FLOAT64 = 10
};

int bytes_of(int dt) {
    switch (dt) {
        case DT_UINT8: case DT_INT8: return 1;
        case DT_UINT16: case DT_INT16: return 2;
        case DT_UINT32: case DT_INT32: case DT_FLOAT32: return 4;
        case DT_UINT64: case DT_INT64: case DT_FLOAT64: return 8;
        default: return 0;
    }
}

// Kernel input kind for a reference data type. The reference reads bit depth
// <= 8 as uint8, <= 16 as uint16 and everything wider as uint32
// (cpu_kernels.tpp:35-53). 64-bit types are not supported.
int input_kind(int dt, bool float_as_uint) {
    switch (dt) {
        case DT_UINT8: case DT_INT8: return IN_U8;
        case DT_UINT16: case DT_INT16: return IN_U16;
        case DT_UINT32: case DT_INT32: return IN_U32;
        case DT_FLOAT32: return float_as_uint ? IN_U32 : IN_F32;
        default: return -1;
    }
}

struct TableSlot {
    int2* lin = nullptr;
    int2* cub = nullptr;
    int* lzb = nullptr;
    float* lzw = nullptr;
    float2* wph = nullptr;
    float2* dcr = nullptr;  // DC response for the exact DC split (n/2)
    bool has_dcr = false;
    cudaEvent_t last_use = nullptr;
};

}  // namespace

struct ope_b200_ctx {
    ope_b200_config cfg{};
    int n = 0;
    long long m = 0;  // A-scans per buffer
    int in_kind = 0;
    int interp = INTERP_NONE;
    size_t in_bytes = 0, out_bytes = 0;
    int device = 0;
    cudaStream_t stream = nullptr;

    std::vector<float> resample, window, cos_sin;
    bool tables_dirty = true;
    TableSlot slot[2];
    int active = -1;
    float2* d_tw = nullptr;
    int* d_status = nullptr;

    // fixed-pattern noise
    FpnState fpn;

    // post-process background (profile on the device; the host copy is
    // refreshed lazily after a recording)
    std::vector<float> bg_profile;
    bool bg_record_requested = false;
    float* d_bg = nullptr;   // profile, n/2
    float* d_bgv = nullptr;  // weight * profile + offset, n/2
    bool bg_valid = false, bgv_dirty = true, bg_host_stale = false;

    // sinusoidal scan correction: curve (A-scans per B-scan) and scratch image
    float* d_sin_curve = nullptr;
    float* d_sin_tmp = nullptr;
    size_t sin_tmp_bytes = 0;
    cudaEvent_t ev_sin = nullptr;  // last use of the scratch image (frames on other streams wait for it)
    bool ev_sin_recorded = false;

    // host-path buffers
    void* d_in = nullptr;
    float* d_out = nullptr;

    // pipelined host path (ope_b200_process_host)
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
    cudaEvent_t ev_pipe[128] = {};

    // test hook: next launch skips its first bulk copy and waits at most this long
    unsigned long long inject_stall_ns = 0;
    bool inject_wait_abort = false;

    // streaming ring (ope_b200_submit / wait / release)
    struct RingSlot {
        cudaStream_t stream = nullptr;
        void* d_in = nullptr;
        float* d_out = nullptr;
        float* h_out = nullptr;  // pinned
        float* h_dst = nullptr;  // where this frame's output lands (h_out or the caller's buffer)
        cudaEvent_t ev_in = nullptr, ev_done = nullptr;
        uint64_t ticket = 0;
        bool busy = false;
    };
    std::vector<RingSlot> ring;
    uint64_t next_ticket = 1;
    cudaEvent_t ev_last_compute = nullptr;

    std::string err;
    std::mutex mu;
};

namespace {

int fail(ope_b200_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(ope_b200_ctx* c, cudaError_t e, const char* what) {
    return fail(c, OPE_B200_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define OPE_CU(ctx, call)                                         \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);  \
    } while (0)

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int validate_cfg(const ope_b200_config* c, std::string* why) {
    if (!c) { *why = "null configuration"; return OPE_B200_E_INVALID; }
    if (c->signal_length <= 0 || c->ascans_per_bscan <= 0 || c->bscans_per_buffer <= 0) {
        *why = "invalid processor configuration (non-positive dimension)";
        return OPE_B200_E_INVALID;
    }
    if (!chain_length_supported(c->signal_length)) {
        *why = "signal length " + std::to_string(c->signal_length) +
               " unsupported: the B200 chain needs a power of two in [512, 8192]";
        return OPE_B200_E_UNSUPPORTED;
    }
    if (input_kind(c->input_dtype, c->float32_as_uint32 != 0) < 0) {
        *why = "input data type " + std::to_string(c->input_dtype) + " unsupported";
        return OPE_B200_E_UNSUPPORTED;
    }
    if (c->resampling_enabled && (c->interpolation < 0 || c->interpolation > 2)) {
        *why = "unknown interpolation method";
        return OPE_B200_E_INVALID;
    }
    if (c->dc_removal_enabled && c->dc_window <= 0) {
        *why = "rolling-average window must be >= 1";
        return OPE_B200_E_INVALID;
    }
    if (c->fpn_bscan_count < 1) {
        *why = "fixedPatternNoiseBscanCount must be >= 1";
        return OPE_B200_E_INVALID;
    }
    return OPE_B200_OK;
}

void free_slot(TableSlot& s) {
    cudaFree(s.lin);
    cudaFree(s.cub);
    cudaFree(s.lzb);
    cudaFree(s.lzw);
    cudaFree(s.wph);
    cudaFree(s.dcr);
    if (s.last_use) cudaEventDestroy(s.last_use);
    s = TableSlot{};
}

// Builds the device tables from the current curves into the inactive slot.
int rebuild_tables(ope_b200_ctx* c) {
    const int n = c->n;
    const auto& cfg = c->cfg;
    const int target = (c->active == 0) ? 1 : 0;
    TableSlot& s = c->slot[target];
    OPE_CU(c, cudaEventSynchronize(s.last_use));  // no in-flight launch still reads this slot

    // resampling
    c->interp = INTERP_NONE;
    std::vector<float> lz_w;
    if (cfg.resampling_enabled) {
        if (c->resample.size() != static_cast<size_t>(n))
            return fail(c, OPE_B200_E_STATE, "resampling enabled but no curve of length N was set");
        const int method = cfg.interpolation;
        if (method == 0) {
            std::vector<int2> tab = build_linear_table(c->resample.data(), n);
            OPE_CU(c, cudaMemcpy(s.lin, tab.data(), n * sizeof(int2), cudaMemcpyHostToDevice));
            c->interp = INTERP_LINEAR;
        } else if (method == 1) {
            std::vector<int2> tab = build_cubic_table(c->resample.data(), n);
            OPE_CU(c, cudaMemcpy(s.cub, tab.data(), n * sizeof(int2), cudaMemcpyHostToDevice));
            c->interp = INTERP_CUBIC;
        } else {
            std::vector<int> base;
            build_lanczos_table(c->resample.data(), n, base, lz_w);
            std::vector<float>& w = lz_w;
            OPE_CU(c, cudaMemcpy(s.lzb, base.data(), n * sizeof(int), cudaMemcpyHostToDevice));
            OPE_CU(c, cudaMemcpy(s.lzw, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
            c->interp = INTERP_LANCZOS;
        }
    }

    // window x phase: a disabled stage multiplies by exactly 1 (cos 1, sin 0)
    const bool win = cfg.windowing_enabled && c->window.size() == static_cast<size_t>(n);
    if (cfg.windowing_enabled && !win)
        return fail(c, OPE_B200_E_STATE, "windowing enabled but no window curve of length N was set");
    // dispersionCompensation skips when the phase length differs from N (cpu_kernels.tpp:205-208)
    const bool disp = cfg.dispersion_enabled && c->cos_sin.size() == 2 * static_cast<size_t>(n);
    std::vector<float2> wph = build_window_phase(win ? c->window.data() : nullptr, disp ? c->cos_sin.data() : nullptr, n);
    OPE_CU(c, cudaMemcpy(s.wph, wph.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    // exact DC split: not needed when the rolling-average DC removal is on
    s.has_dcr = cfg.dc_split && !cfg.dc_removal_enabled;
    if (s.has_dcr) {
        std::vector<float2> d = build_dc_response(n, c->interp, lz_w.empty() ? nullptr : lz_w.data(),
                                                  win ? c->window.data() : nullptr,
                                                  disp ? c->cos_sin.data() : nullptr);
        OPE_CU(c, cudaMemcpy(s.dcr, d.data(), (n / 2) * sizeof(float2), cudaMemcpyHostToDevice));
    }
    c->active = target;
    c->tables_dirty = false;
    return OPE_B200_OK;
}

int alloc_slot(ope_b200_ctx* c, TableSlot& s) {
    const size_t n = static_cast<size_t>(c->n);
    OPE_CU(c, cudaMalloc(&s.lin, n * sizeof(int2)));
    OPE_CU(c, cudaMalloc(&s.cub, n * sizeof(int2)));
    OPE_CU(c, cudaMalloc(&s.lzb, n * sizeof(int)));
    OPE_CU(c, cudaMalloc(&s.lzw, 16 * n * sizeof(float)));
    OPE_CU(c, cudaMalloc(&s.wph, n * sizeof(float2)));
    OPE_CU(c, cudaMalloc(&s.dcr, (n / 2) * sizeof(float2)));
    OPE_CU(c, cudaEventCreateWithFlags(&s.last_use, cudaEventDisableTiming));
    return OPE_B200_OK;
}

}  // namespace

namespace ope_b200 {
bool chain_length_supported(int n) { return n >= 512 && n <= 8192 && (n & (n - 1)) == 0; }
}  // namespace ope_b200

// Builds kernel arguments for the current configuration; tables must be valid.
static ChainArgs make_args(ope_b200_ctx* c, const void* d_in, float* d_out, long long m, const float2* fpn) {
    ChainArgs a{};
    a.in = d_in;
    a.out = d_out;
    a.m = m;
    a.tw = c->d_tw;
    const TableSlot& s = c->slot[c->active];
    a.lin = s.lin;
    a.cub = s.cub;
    a.lz_base = s.lzb;
    a.lz_w = s.lzw;
    a.wph = s.wph;
    a.fpn = fpn;
    a.dc_window = c->cfg.dc_removal_enabled ? c->cfg.dc_window : 0;
    a.dc_ref_order = c->cfg.dc_reference_order ? 1 : 0;
    const auto& cf = c->cfg;
    scaling_constants(cf.log_scaling != 0, cf.grayscale_min, cf.grayscale_max, cf.addend, cf.multiplicator, c->n, a);
    a.flip = c->cfg.bscan_flip ? 1 : 0;
    a.ascans_per_bscan = c->cfg.ascans_per_bscan;
    a.bscans = static_cast<int>((m + c->cfg.ascans_per_bscan - 1) / c->cfg.ascans_per_bscan);
    a.status = c->d_status;
    a.timeout_ns = 2000000000ull;
    a.neg_zero = -0.0f;
    a.dc_resp = s.has_dcr ? s.dcr : nullptr;
    // 8/16-bit samples only; 32-bit samples ignore the flag, as the reference CPU backend does
    a.bitshift = (c->cfg.bitshift && (c->in_kind == IN_U8 || c->in_kind == IN_U16)) ? 1 : 0;
    return a;
}

namespace ope_b200 {

// Chain arguments of the context's current configuration for the batched
// launcher (batch.cu): tables rebuilt if a curve changed, the fixed-pattern
// profile if subtraction is on. Input, output and A-scan count are left for
// the caller. FPN determination needs the per-buffer state machine of
// process_locked and is not available to batches.
int ctx_batch_args(ope_b200_ctx* c, ChainArgs* a, int* n, int* in_kind, int* interp, int* device) {
    if (!c || !a) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    OPE_CU(c, cudaSetDevice(c->device));
    if (c->tables_dirty) {
        int rc = rebuild_tables(c);
        if (rc != OPE_B200_OK) return rc;
    }
    if (c->fpn.requested || c->cfg.fpn_continuous)
        return fail(c, OPE_B200_E_UNSUPPORTED, "FPN determination is not available in a batch");
    if (c->cfg.sinusoidal_correction)
        return fail(c, OPE_B200_E_UNSUPPORTED, "sinusoidal scan correction is not available in a batch");
    const float2* fpn = (c->cfg.fpn_removal && c->fpn.valid) ? c->fpn.d_profile : nullptr;
    *a = make_args(c, nullptr, nullptr, 0, fpn);
    if (c->cfg.post_bg_removal) {
        if (c->bg_record_requested)
            return fail(c, OPE_B200_E_UNSUPPORTED, "post-process background recording is not available in a batch");
        if (c->bg_valid) {
            if (c->bgv_dirty) {
                OPE_CU(c, bg_values(c->d_bg, c->n / 2, c->cfg.bg_weight, c->cfg.bg_offset, c->d_bgv, nullptr));
                OPE_CU(c, cudaDeviceSynchronize());
                c->bgv_dirty = false;
            }
            a->bgv = c->d_bgv;
        }
    }
    *n = c->n;
    *in_kind = c->in_kind;
    *interp = c->interp;
    *device = c->device;
    return OPE_B200_OK;
}

const char* ctx_error(const ope_b200_ctx* c) { return c ? c->err.c_str() : "null context"; }

}  // namespace ope_b200

extern "C" {

int ope_b200_abi_version(void) { return OPE_B200_ABI_VERSION; }

int ope_b200_device_supported(int32_t device) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return 0;
    return p.major == 10 ? 1 : 0;
}

void ope_b200_config_default(ope_b200_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->signal_length = 1024;
    c->ascans_per_bscan = 512;
    c->bscans_per_buffer = 1;
    c->input_dtype = DT_UINT16;
    c->interpolation = 0;
    c->dc_window = 64;
    c->log_scaling = 1;
    c->grayscale_min = 30.0f;
    c->grayscale_max = 100.0f;
    c->addend = 0.0f;
    c->multiplicator = 1.0f;
    c->fpn_bscan_count = 1;
    c->bg_weight = 1.0f;
    c->bg_offset = 0.0f;
    c->num_input_buffers = 2;
    c->dc_split = 1;
}

// why the calling thread's last ope_b200_create failed (ope_b200_last_error(NULL))
static thread_local std::string t_create_err;

int ope_b200_create(const ope_b200_config* cfg, ope_b200_ctx** out) {
    if (!out) return OPE_B200_E_INVALID;
    *out = nullptr;
    t_create_err.clear();
    std::string why;
    int rc = validate_cfg(cfg, &why);
    if (rc != OPE_B200_OK) {
        t_create_err = why;
        std::fprintf(stderr, "ope_b200_create: %s\n", why.c_str());
        return rc;
    }
    auto* c = new ope_b200_ctx();
    c->cfg = *cfg;
    c->n = cfg->signal_length;
    c->m = static_cast<long long>(cfg->ascans_per_bscan) * cfg->bscans_per_buffer;
    c->in_kind = input_kind(cfg->input_dtype, cfg->float32_as_uint32 != 0);
    c->in_bytes = static_cast<size_t>(c->m) * c->n * bytes_of(cfg->input_dtype);
    c->out_bytes = static_cast<size_t>(c->m) * (c->n / 2) * sizeof(float);
    c->device = cfg->device;
    auto bail = [&](int code) {
        cudaError_t e = cudaGetLastError();
        t_create_err = std::string("device set-up failed on device ") + std::to_string(c->device) + ": " +
                       cudaGetErrorString(e);
        ope_b200_destroy(c);
        return code;
    };
    if (cudaSetDevice(c->device) != cudaSuccess) return bail(OPE_B200_E_CUDA);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(OPE_B200_E_CUDA);
    for (auto& s : c->slot)
        if (alloc_slot(c, s) != OPE_B200_OK) return bail(OPE_B200_E_CUDA);
    std::vector<float2> tw = build_twiddles(c->n);
    if (cudaMalloc(&c->d_tw, c->n * sizeof(float2)) != cudaSuccess) return bail(OPE_B200_E_NOMEM);
    if (cudaMemcpy(c->d_tw, tw.data(), c->n * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(OPE_B200_E_CUDA);
    if (cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess) return bail(OPE_B200_E_NOMEM);
    if (cudaMemset(c->d_status, 0, sizeof(int)) != cudaSuccess) return bail(OPE_B200_E_CUDA);
    if (fpn_init(c->fpn, c->n) != cudaSuccess) return bail(OPE_B200_E_NOMEM);
    *out = c;
    return OPE_B200_OK;
}

void ope_b200_destroy(ope_b200_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& r : c->ring) {
        if (r.stream) cudaStreamSynchronize(r.stream);
        cudaFree(r.d_in);
        cudaFree(r.d_out);
        cudaFreeHost(r.h_out);
        if (r.ev_in) cudaEventDestroy(r.ev_in);
        if (r.ev_done) cudaEventDestroy(r.ev_done);
        if (r.stream) cudaStreamDestroy(r.stream);
    }
    if (c->ev_last_compute) cudaEventDestroy(c->ev_last_compute);
    if (c->s_h2d) {
        cudaStreamSynchronize(c->s_h2d);
        cudaStreamDestroy(c->s_h2d);
    }
    if (c->s_d2h) {
        cudaStreamSynchronize(c->s_d2h);
        cudaStreamDestroy(c->s_d2h);
    }
    for (auto& e : c->ev_pipe)
        if (e) cudaEventDestroy(e);
    for (auto& s : c->slot) free_slot(s);
    cudaFree(c->d_tw);
    cudaFree(c->d_status);
    cudaFree(c->d_in);
    cudaFree(c->d_out);
    fpn_free(c->fpn);
    cudaFree(c->d_bg);
    cudaFree(c->d_bgv);
    cudaFree(c->d_sin_curve);
    cudaFree(c->d_sin_tmp);
    if (c->ev_sin) cudaEventDestroy(c->ev_sin);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* ope_b200_last_error(const ope_b200_ctx* c) {
    if (c) return c->err.c_str();
    return t_create_err.empty() ? "null context" : t_create_err.c_str();
}

int ope_b200_update_config(ope_b200_ctx* c, const ope_b200_config* cfg) {
    if (!c || !cfg) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    std::string why;
    int rc = validate_cfg(cfg, &why);
    if (rc != OPE_B200_OK) return fail(c, rc, why);
    if (cfg->signal_length != c->cfg.signal_length || cfg->ascans_per_bscan != c->cfg.ascans_per_bscan ||
        cfg->bscans_per_buffer != c->cfg.bscans_per_buffer || cfg->device != c->cfg.device)
        return fail(c, OPE_B200_E_STATE, "dimension change requires a new context");
    const bool dt_change = cfg->input_dtype != c->cfg.input_dtype || cfg->float32_as_uint32 != c->cfg.float32_as_uint32;
    c->cfg = *cfg;
    c->bgv_dirty = true;  // background weight or offset may have changed
    if (dt_change) {
        c->in_kind = input_kind(cfg->input_dtype, cfg->float32_as_uint32 != 0);
        c->in_bytes = static_cast<size_t>(c->m) * c->n * bytes_of(cfg->input_dtype);
        cudaFree(c->d_in);
        c->d_in = nullptr;
    }
    c->tables_dirty = true;
    return OPE_B200_OK;
}

int ope_b200_set_resampling_curve(ope_b200_ctx* c, const float* curve, size_t n) {
    if (!c) return OPE_B200_E_INVALID;
    if (!curve && n > 0) return fail(c, OPE_B200_E_INVALID, "Invalid resampling curve pointer");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resample.assign(curve, curve + n);
    c->tables_dirty = true;
    return OPE_B200_OK;
}

int ope_b200_set_window_curve(ope_b200_ctx* c, const float* curve, size_t n) {
    if (!c) return OPE_B200_E_INVALID;
    if (!curve && n > 0) return fail(c, OPE_B200_E_INVALID, "Invalid window curve pointer");
    std::lock_guard<std::mutex> lk(c->mu);
    c->window.assign(curve, curve + n);
    c->tables_dirty = true;
    return OPE_B200_OK;
}

int ope_b200_set_dispersion_curve(ope_b200_ctx* c, const float* cs, size_t n_floats) {
    if (!c) return OPE_B200_E_INVALID;
    if (!cs && n_floats > 0) return fail(c, OPE_B200_E_INVALID, "Invalid dispersion curve pointer");
    std::lock_guard<std::mutex> lk(c->mu);
    c->cos_sin.assign(cs, cs + (n_floats / 2) * 2);
    c->tables_dirty = true;
    return OPE_B200_OK;
}

static int process_locked(ope_b200_ctx* c, const void* d_in, void* d_out, long long m, cudaStream_t s,
                          bool bins = false) {
    if (!d_in || !d_out || m < 1) return fail(c, OPE_B200_E_INVALID, "null buffer or empty A-scan count");
    if (!aligned16(d_in)) return fail(c, OPE_B200_E_INVALID, "input buffer must be 16-byte aligned");
    if ((reinterpret_cast<uintptr_t>(d_out) & (bins ? 7u : 3u)) != 0)
        return fail(c, OPE_B200_E_INVALID, "output buffer is not aligned to its element size");
    OPE_CU(c, cudaSetDevice(c->device));
    if (c->tables_dirty) {
        int rc = rebuild_tables(c);
        if (rc != OPE_B200_OK) return rc;
    }
    // fixed-pattern noise: determination (statistics pass + finalize) before
    // the frame that uses it, as computeFixedPatternNoiseIfRequested runs
    // before the subtraction loop (cpu_backend.cpp:245-255)
    const float2* fpn = nullptr;
    if (c->cfg.fpn_removal || c->fpn.requested || c->cfg.fpn_continuous) {
        ChainArgs a = make_args(c, d_in, nullptr, m, nullptr);
        int rc = fpn_process_frame(c->fpn, c->cfg, c->in_kind, c->interp, a, s, &c->err);
        if (rc != OPE_B200_OK) return rc;
        if (c->cfg.fpn_removal && c->fpn.valid) fpn = c->fpn.d_profile;
    }
    ChainArgs a = make_args(c, d_in, bins ? nullptr : static_cast<float*>(d_out), m, fpn);
    if (bins) a.bins_out = static_cast<float2*>(d_out);
    // post-process background (cpu_backend.cpp:283-301): a recording frame is
    // scaled first, its mean A-scan becomes the profile, then it is subtracted;
    // other frames subtract the profile in the chain epilogue
    const int half = c->n / 2;
    const bool bg_on = c->cfg.post_bg_removal && !bins;
    const bool record = bg_on && c->bg_record_requested;
    if (bg_on && (record || c->bg_valid)) {
        if (!c->d_bg) OPE_CU(c, cudaMalloc(&c->d_bg, half * sizeof(float)));
        if (!c->d_bgv) OPE_CU(c, cudaMalloc(&c->d_bgv, half * sizeof(float)));
        // frames still in flight on other streams may read the current values:
        // a recording or a changed weight/offset waits for them (rare events)
        if (record || (c->bg_valid && c->bgv_dirty)) OPE_CU(c, cudaDeviceSynchronize());
    }
    if (bg_on && !record && c->bg_valid && c->bgv_dirty) {
        OPE_CU(c, bg_values(c->d_bg, half, c->cfg.bg_weight, c->cfg.bg_offset, c->d_bgv, s));
        c->bgv_dirty = false;
    }
    const float* bgv_now = (bg_on && !record && c->bg_valid) ? c->d_bgv : nullptr;
    // sinusoidal scan correction (cuda_backend.cu:696-706, after the flip and
    // before the background): the chain writes a scratch image, the correction
    // interpolates across A-scans into the output and subtracts the background
    const bool sin_on = c->cfg.sinusoidal_correction && !bins;
    if (sin_on) {
        const size_t need = static_cast<size_t>(m) * half * sizeof(float);
        if (need > c->sin_tmp_bytes) {
            OPE_CU(c, cudaStreamSynchronize(s));
            cudaFree(c->d_sin_tmp);
            c->d_sin_tmp = nullptr;
            c->sin_tmp_bytes = 0;
            OPE_CU(c, cudaMalloc(&c->d_sin_tmp, need));
            c->sin_tmp_bytes = need;
        }
        if (!c->d_sin_curve) {
            OPE_CU(c, cudaMalloc(&c->d_sin_curve, c->cfg.ascans_per_bscan * sizeof(float)));
            OPE_CU(c, sin_curve(c->d_sin_curve, c->cfg.ascans_per_bscan, s));
        }
        if (!c->ev_sin) OPE_CU(c, cudaEventCreateWithFlags(&c->ev_sin, cudaEventDisableTiming));
        // one scratch image per context: a frame on another stream (the ring)
        // must have finished its correction before this chain overwrites it
        if (c->ev_sin_recorded) OPE_CU(c, cudaStreamWaitEvent(s, c->ev_sin, 0));
        a.out = c->d_sin_tmp;
    } else {
        a.bgv = bgv_now;
    }
    if (c->inject_stall_ns) {
        a.debug_skip_first_copy = 1;
        a.timeout_ns = c->inject_stall_ns;
        c->inject_stall_ns = 0;
    }
    if (c->inject_wait_abort) {
        a.debug_abort_first_wait = 1;
        c->inject_wait_abort = false;
    }
    cudaError_t e = launch_chain(c->n, c->in_kind, c->interp, a, s, 0, nullptr);
    if (e != cudaSuccess) return cuda_fail(c, e, "chain launch");
    OPE_CU(c, cudaEventRecord(c->slot[c->active].last_use, s));
    if (sin_on) {
        OPE_CU(c, sin_correct(static_cast<float*>(d_out), c->d_sin_tmp, c->d_sin_curve, half,
                              c->cfg.ascans_per_bscan, m, bgv_now, s));
        OPE_CU(c, cudaEventRecord(c->ev_sin, s));
        c->ev_sin_recorded = true;
    }
    if (record) {
        float* out = static_cast<float*>(d_out);
        OPE_CU(c, bg_record(out, m, half, c->d_bg, s));
        OPE_CU(c, bg_values(c->d_bg, half, c->cfg.bg_weight, c->cfg.bg_offset, c->d_bgv, s));
        OPE_CU(c, bg_subtract(out, m, half, c->d_bgv, s));
        c->bg_valid = true;
        c->bgv_dirty = false;
        c->bg_host_stale = true;
        c->bg_record_requested = false;
    }
    return OPE_B200_OK;
}

int ope_b200_process_device_n(ope_b200_ctx* c, const void* d_in, float* d_out, int64_t m, void* stream) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    return process_locked(c, d_in, d_out, m, static_cast<cudaStream_t>(stream));
}

int ope_b200_process_bins_device(ope_b200_ctx* c, const void* d_in, void* d_bins, int64_t m, void* stream) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    return process_locked(c, d_in, d_bins, m, static_cast<cudaStream_t>(stream), true);
}

int ope_b200_test_inject_copy_stall(ope_b200_ctx* c, uint32_t timeout_us) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    c->inject_stall_ns = static_cast<unsigned long long>(timeout_us ? timeout_us : 1) * 1000ull;
    return OPE_B200_OK;
}

int ope_b200_test_inject_wait_abort(ope_b200_ctx* c) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    c->inject_wait_abort = true;
    return OPE_B200_OK;
}

int ope_b200_process_device(ope_b200_ctx* c, const void* d_in, float* d_out, void* stream) {
    if (!c) return OPE_B200_E_INVALID;
    return ope_b200_process_device_n(c, d_in, d_out, c->m, stream);
}

int ope_b200_process_host(ope_b200_ctx* c, const void* h_in, float* h_out) {
    if (!c) return OPE_B200_E_INVALID;
    if (!h_in || !h_out) return fail(c, OPE_B200_E_INVALID, "null host buffer");
    std::lock_guard<std::mutex> lk(c->mu);
    OPE_CU(c, cudaSetDevice(c->device));
    if (!c->d_in) OPE_CU(c, cudaMalloc(&c->d_in, c->in_bytes));
    if (!c->d_out) OPE_CU(c, cudaMalloc(&c->d_out, c->out_bytes));
    // Pipelined in chunks of whole B-scan pairs: the copy in of chunk k+1 and
    // the copy out of chunk k-1 (two copy engines) overlap the chain on chunk
    // k. Chunks start at even B-scans so the B-scan flip sees the same
    // parities; FPN determination needs the whole buffer and runs unchunked.
    const long long A = c->cfg.ascans_per_bscan;
    const long long B = c->cfg.bscans_per_buffer;
    // 16 chunks: measured 6.28 ms per 2048 x 1024 x 64 uint16 buffer (4: 6.88,
    // 8: 6.36, 32: 6.52) against 5.64 ms for the bare concurrent copies
    const long long kChunks = 16;
    const long long bs_per_chunk = 2 * ((B + 2 * kChunks - 1) / (2 * kChunks));
    const bool chunked = !(c->fpn.requested || c->cfg.fpn_continuous) &&
                         !(c->cfg.post_bg_removal && c->bg_record_requested) && !c->cfg.sinusoidal_correction &&
                         B >= 4;
    if (!chunked) {
        OPE_CU(c, cudaMemcpyAsync(c->d_in, h_in, c->in_bytes, cudaMemcpyHostToDevice, c->stream));
        int rc = process_locked(c, c->d_in, c->d_out, c->m, c->stream);
        if (rc != OPE_B200_OK) return rc;
        OPE_CU(c, cudaMemcpyAsync(h_out, c->d_out, c->out_bytes, cudaMemcpyDeviceToHost, c->stream));
        OPE_CU(c, cudaStreamSynchronize(c->stream));
    } else {
        if (!c->s_h2d) OPE_CU(c, cudaStreamCreateWithFlags(&c->s_h2d, cudaStreamNonBlocking));
        if (!c->s_d2h) OPE_CU(c, cudaStreamCreateWithFlags(&c->s_d2h, cudaStreamNonBlocking));
        for (int k = 0; k < 2 * kChunks; ++k)
            if (!c->ev_pipe[k]) OPE_CU(c, cudaEventCreateWithFlags(&c->ev_pipe[k], cudaEventDisableTiming));
        const size_t in_row = c->in_bytes / static_cast<size_t>(c->m);
        const size_t out_row = static_cast<size_t>(c->n / 2) * sizeof(float);
        int k = 0;
        for (long long b0 = 0; b0 < B; b0 += bs_per_chunk, ++k) {
            const long long r0 = b0 * A;
            const long long rows = std::min(bs_per_chunk, B - b0) * A;
            const unsigned char* src = static_cast<const unsigned char*>(h_in) + r0 * in_row;
            unsigned char* din = static_cast<unsigned char*>(c->d_in) + r0 * in_row;
            float* dout = c->d_out + r0 * (c->n / 2);
            OPE_CU(c, cudaMemcpyAsync(din, src, rows * in_row, cudaMemcpyHostToDevice, c->s_h2d));
            OPE_CU(c, cudaEventRecord(c->ev_pipe[2 * k], c->s_h2d));
            OPE_CU(c, cudaStreamWaitEvent(c->stream, c->ev_pipe[2 * k], 0));
            int rc = process_locked(c, din, dout, rows, c->stream);
            if (rc != OPE_B200_OK) {
                cudaStreamSynchronize(c->s_h2d);
                cudaStreamSynchronize(c->s_d2h);
                return rc;
            }
            OPE_CU(c, cudaEventRecord(c->ev_pipe[2 * k + 1], c->stream));
            OPE_CU(c, cudaStreamWaitEvent(c->s_d2h, c->ev_pipe[2 * k + 1], 0));
            OPE_CU(c, cudaMemcpyAsync(h_out + r0 * (c->n / 2), dout, rows * out_row, cudaMemcpyDeviceToHost, c->s_d2h));
        }
        OPE_CU(c, cudaStreamSynchronize(c->s_d2h));
        OPE_CU(c, cudaStreamSynchronize(c->stream));
    }
    int st = 0;
    OPE_CU(c, cudaMemcpy(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != 0) {
        cudaMemset(c->d_status, 0, sizeof(int));
        return fail(c, OPE_B200_E_DEVICE, "kernel reported status " + std::to_string(st));
    }
    return OPE_B200_OK;
}

int ope_b200_synchronize(ope_b200_ctx* c, int32_t* device_status) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    OPE_CU(c, cudaSetDevice(c->device));
    OPE_CU(c, cudaDeviceSynchronize());
    int st = 0;
    OPE_CU(c, cudaMemcpy(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    OPE_CU(c, cudaMemset(c->d_status, 0, sizeof(int)));
    if (device_status) *device_status = st;
    return OPE_B200_OK;
}

int ope_b200_request_fpn_determination(ope_b200_ctx* c) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    c->fpn.requested = true;
    return OPE_B200_OK;
}

int ope_b200_set_fpn_profile(ope_b200_ctx* c, const float* p, size_t pairs) {
    if (!c) return OPE_B200_E_INVALID;
    if (!p && pairs > 0) return fail(c, OPE_B200_E_INVALID, "Invalid fixed-pattern noise profile pointer");
    std::lock_guard<std::mutex> lk(c->mu);
    OPE_CU(c, cudaSetDevice(c->device));
    return fpn_set_profile(c->fpn, p, pairs, c->stream, &c->err);
}

int ope_b200_get_fpn_profile(ope_b200_ctx* c, float* out, size_t cap_pairs, size_t* pairs) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    OPE_CU(c, cudaSetDevice(c->device));
    return fpn_get_profile(c->fpn, out, cap_pairs, pairs, &c->err);
}

int ope_b200_request_bg_recording(ope_b200_ctx* c) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    c->bg_record_requested = true;
    return OPE_B200_OK;
}

int ope_b200_set_bg_profile(ope_b200_ctx* c, const float* p, size_t n) {
    if (!c) return OPE_B200_E_INVALID;
    if (!p) return fail(c, OPE_B200_E_INVALID, "Background curve data is null");
    std::lock_guard<std::mutex> lk(c->mu);
    if (n != static_cast<size_t>(c->n / 2))
        return fail(c, OPE_B200_E_INVALID, "Invalid background buffer size. Expected " + std::to_string(c->n / 2) +
                                               " but got " + std::to_string(n));
    c->bg_profile.assign(p, p + n);
    OPE_CU(c, cudaSetDevice(c->device));
    if (!c->d_bg) OPE_CU(c, cudaMalloc(&c->d_bg, n * sizeof(float)));
    if (!c->d_bgv) OPE_CU(c, cudaMalloc(&c->d_bgv, n * sizeof(float)));
    OPE_CU(c, cudaDeviceSynchronize());  // no frame in flight still reads the old values
    OPE_CU(c, cudaMemcpy(c->d_bg, p, n * sizeof(float), cudaMemcpyHostToDevice));
    c->bg_valid = true;
    c->bgv_dirty = true;
    c->bg_host_stale = false;
    return OPE_B200_OK;
}

int ope_b200_get_bg_profile(ope_b200_ctx* c, float* out, size_t cap, size_t* n) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->bg_host_stale) {  // recorded on the device since the last read
        OPE_CU(c, cudaSetDevice(c->device));
        OPE_CU(c, cudaDeviceSynchronize());
        c->bg_profile.resize(c->n / 2);
        OPE_CU(c, cudaMemcpy(c->bg_profile.data(), c->d_bg, c->bg_profile.size() * sizeof(float),
                             cudaMemcpyDeviceToHost));
        c->bg_host_stale = false;
    }
    if (n) *n = c->bg_profile.size();
    if (out) std::memcpy(out, c->bg_profile.data(), std::min(cap, c->bg_profile.size()) * sizeof(float));
    return OPE_B200_OK;
}

}  // extern "C"

namespace ope_b200 {

cudaError_t launch_chain(int n, int in_kind, int interp, const ChainArgs& a, cudaStream_t s, int max_ctas,
                         LaunchInfo* info) {
    switch (n) {
        case 512: return launch_chain_n512(in_kind, interp, a, s, max_ctas, info);
        case 1024: return launch_chain_n1024(in_kind, interp, a, s, max_ctas, info);
        case 2048: return launch_chain_n2048(in_kind, interp, a, s, max_ctas, info);
        case 4096: return launch_chain_n4096(in_kind, interp, a, s, max_ctas, info);
        case 8192: return launch_chain_n8192(in_kind, interp, a, s, max_ctas, info);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ope_b200

// ---------------------------------------------------------------------------
// Streaming ring: the IOBuffer path of ProcessingBackend::process
// (backend_interface.h:24,35-37). Each of num_input_buffers slots owns a
// stream, device input/output buffers and a pinned host output buffer. A frame
// is H2D -> chain -> D2H on its slot's stream; the chain of frame i+1 waits for
// the chain of frame i (FPN state is shared and ordered), so copies of
// neighbouring frames overlap the computation in both directions.
// ---------------------------------------------------------------------------

namespace {

bool wait_event_bounded(cudaEvent_t ev, int timeout_ms, cudaError_t* err) {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    while (true) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return true;
        if (e != cudaErrorNotReady) {
            *err = e;
            return false;
        }
        if (timeout_ms >= 0 &&
            std::chrono::duration_cast<std::chrono::milliseconds>(clk::now() - t0).count() > timeout_ms) {
            *err = cudaErrorNotReady;
            return false;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

int ensure_ring(ope_b200_ctx* c) {
    if (!c->ring.empty()) return OPE_B200_OK;
    const int depth = c->cfg.num_input_buffers >= 2 ? c->cfg.num_input_buffers : 2;
    c->ring.resize(depth);
    for (auto& r : c->ring) {
        OPE_CU(c, cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking));
        OPE_CU(c, cudaMalloc(&r.d_in, c->in_bytes));
        OPE_CU(c, cudaMalloc(&r.d_out, c->out_bytes));
        OPE_CU(c, cudaHostAlloc(reinterpret_cast<void**>(&r.h_out), c->out_bytes, cudaHostAllocPortable));
        OPE_CU(c, cudaEventCreateWithFlags(&r.ev_in, cudaEventDisableTiming));
        OPE_CU(c, cudaEventCreateWithFlags(&r.ev_done, cudaEventDisableTiming));
    }
    OPE_CU(c, cudaEventCreateWithFlags(&c->ev_last_compute, cudaEventDisableTiming));
    return OPE_B200_OK;
}

ope_b200_ctx::RingSlot* find_slot(ope_b200_ctx* c, uint64_t ticket) {
    if (c->ring.empty() || ticket == 0) return nullptr;
    auto& r = c->ring[(ticket - 1) % c->ring.size()];
    return (r.busy && r.ticket == ticket) ? &r : nullptr;
}

}  // namespace

extern "C" {

int ope_b200_ring_depth(ope_b200_ctx* c) {
    if (!c) return OPE_B200_E_INVALID;
    return c->cfg.num_input_buffers >= 2 ? c->cfg.num_input_buffers : 2;
}

int ope_b200_host_register(void* ptr, size_t bytes) {
    if (!ptr || !bytes) return OPE_B200_E_INVALID;
    return cudaHostRegister(ptr, bytes, cudaHostRegisterPortable) == cudaSuccess ? OPE_B200_OK : OPE_B200_E_CUDA;
}

int ope_b200_host_unregister(void* ptr) {
    if (!ptr) return OPE_B200_E_INVALID;
    return cudaHostUnregister(ptr) == cudaSuccess ? OPE_B200_OK : OPE_B200_E_CUDA;
}

int ope_b200_submit(ope_b200_ctx* c, const void* h_in, uint64_t* ticket) {
    return ope_b200_submit_to(c, h_in, nullptr, ticket);
}

int ope_b200_submit_to(ope_b200_ctx* c, const void* h_in, float* h_out_dst, uint64_t* ticket) {
    if (!c) return OPE_B200_E_INVALID;
    if (!h_in || !ticket) return fail(c, OPE_B200_E_INVALID, "null input buffer or ticket");
    std::lock_guard<std::mutex> lk(c->mu);
    OPE_CU(c, cudaSetDevice(c->device));
    int rc = ensure_ring(c);
    if (rc != OPE_B200_OK) return rc;
    const uint64_t t = c->next_ticket;
    auto& r = c->ring[(t - 1) % c->ring.size()];
    if (r.busy)
        return fail(c, OPE_B200_E_STATE,
                    "all ring slots are in use: release the oldest frame's output before submitting more");
    OPE_CU(c, cudaMemcpyAsync(r.d_in, h_in, c->in_bytes, cudaMemcpyHostToDevice, r.stream));
    OPE_CU(c, cudaEventRecord(r.ev_in, r.stream));
    OPE_CU(c, cudaStreamWaitEvent(r.stream, c->ev_last_compute, 0));
    rc = process_locked(c, r.d_in, r.d_out, c->m, r.stream);
    if (rc != OPE_B200_OK) return rc;
    OPE_CU(c, cudaEventRecord(c->ev_last_compute, r.stream));
    r.h_dst = h_out_dst ? h_out_dst : r.h_out;
    OPE_CU(c, cudaMemcpyAsync(r.h_dst, r.d_out, c->out_bytes, cudaMemcpyDeviceToHost, r.stream));
    OPE_CU(c, cudaEventRecord(r.ev_done, r.stream));
    r.busy = true;
    r.ticket = t;
    c->next_ticket++;
    *ticket = t;
    return OPE_B200_OK;
}

int ope_b200_input_released(ope_b200_ctx* c, uint64_t ticket, int32_t timeout_ms) {
    if (!c) return OPE_B200_E_INVALID;
    cudaEvent_t ev;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        auto* r = find_slot(c, ticket);
        if (!r) return fail(c, OPE_B200_E_INVALID, "unknown or released ticket");
        ev = r->ev_in;
    }
    cudaError_t e = cudaSuccess;
    if (!wait_event_bounded(ev, timeout_ms, &e))
        return e == cudaErrorNotReady ? OPE_B200_E_TIMEOUT : OPE_B200_E_CUDA;
    return OPE_B200_OK;
}

int ope_b200_frame_device_input(ope_b200_ctx* c, uint64_t ticket, void* stream, const void** d_in) {
    if (!c) return OPE_B200_E_INVALID;
    if (!d_in) return fail(c, OPE_B200_E_INVALID, "null output pointer");
    std::lock_guard<std::mutex> lk(c->mu);
    auto* r = find_slot(c, ticket);
    if (!r) return fail(c, OPE_B200_E_INVALID, "unknown or released ticket");
    OPE_CU(c, cudaSetDevice(c->device));
    OPE_CU(c, cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), r->ev_in, 0));
    *d_in = r->d_in;
    return OPE_B200_OK;
}

int ope_b200_wait(ope_b200_ctx* c, uint64_t ticket, int32_t timeout_ms, const float** h_out) {
    if (!c) return OPE_B200_E_INVALID;
    cudaEvent_t ev;
    const float* out;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        auto* r = find_slot(c, ticket);
        if (!r) return fail(c, OPE_B200_E_INVALID, "unknown or released ticket");
        ev = r->ev_done;
        out = r->h_dst;
    }
    cudaError_t e = cudaSuccess;
    if (!wait_event_bounded(ev, timeout_ms, &e)) {
        if (e == cudaErrorNotReady) return OPE_B200_E_TIMEOUT;
        std::lock_guard<std::mutex> lk(c->mu);
        return cuda_fail(c, e, "frame");
    }
    int st = 0;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        OPE_CU(c, cudaMemcpy(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
        if (st != 0) {
            cudaMemset(c->d_status, 0, sizeof(int));
            return fail(c, OPE_B200_E_DEVICE, "kernel reported status " + std::to_string(st));
        }
    }
    if (h_out) *h_out = out;
    return OPE_B200_OK;
}

int ope_b200_release(ope_b200_ctx* c, uint64_t ticket) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    auto* r = find_slot(c, ticket);
    if (!r) return fail(c, OPE_B200_E_INVALID, "unknown or released ticket");
    if (cudaEventQuery(r->ev_done) != cudaSuccess) return fail(c, OPE_B200_E_STATE, "frame still in flight");
    r->busy = false;
    return OPE_B200_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Fixed-pattern-noise determination without device allocation.
//
// Some callers cannot allocate device memory once they are running: a
// real-time acquisition thread must not stall the frame loop (cudaMalloc and
// cudaFree can synchronise the whole device), and integrations that budget all
// device memory at start-up may not allocate afterwards. The allocating path
// (ope_b200_request_fpn_determination + process) grows its partial-sum buffer
// with cudaMalloc on first use. This variant keeps those partial sums and the
// segment accumulators in one file-scope device array of fixed size instead.
// ---------------------------------------------------------------------------

namespace {

constexpr int kNoAllocMaxN = 4096;  // longest A-scan the static scratch serves
constexpr int kNoAllocMaxGx = 8;    // CTAs per FPN segment
constexpr size_t kNoAllocPartial = static_cast<size_t>(FPN_SEGMENTS) * kNoAllocMaxGx * (kNoAllocMaxN / 2) * 3;
constexpr size_t kNoAllocAcc = static_cast<size_t>(FPN_SEGMENTS) * (kNoAllocMaxN / 2) * 3;

// 3.4 MiB per GPU that loads the library, held until the process exits.
static __device__ __align__(256) double g_fpn_noalloc_scratch[kNoAllocPartial + kNoAllocAcc];

// Device address of the scratch array in the current device's context. In host
// code the array's name is only a host-side stand-in, never a device address.
// Looked up on every call (cheap once the module is loaded): an address cached
// across calls would go stale if the host application reset the device and a
// new primary context reloaded the module elsewhere.
cudaError_t noalloc_scratch(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_fpn_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<double*>(p);
    return cudaSuccess;
}

}  // namespace

extern "C" {

int ope_b200_determine_fpn_noalloc(ope_b200_ctx* c, const void* d_in, int64_t num_ascans, float* d_profile,
                                   void* stream) {
    if (!c) return OPE_B200_E_INVALID;
    std::lock_guard<std::mutex> lk(c->mu);
    if (!d_in || !d_profile || num_ascans < 1) return fail(c, OPE_B200_E_INVALID, "null buffer or empty A-scan count");
    if (!aligned16(d_in)) return fail(c, OPE_B200_E_INVALID, "input buffer must be 16-byte aligned");
    if ((reinterpret_cast<uintptr_t>(d_profile) & 7u) != 0)
        return fail(c, OPE_B200_E_INVALID, "profile buffer must be 8-byte aligned");
    if (c->n > kNoAllocMaxN)
        return fail(c, OPE_B200_E_UNSUPPORTED, "no-allocation FPN determination supports signal lengths up to " +
                                                   std::to_string(kNoAllocMaxN));
    const long long required = static_cast<long long>(c->cfg.fpn_bscan_count) * c->cfg.ascans_per_bscan;
    const long long seg_w = required / FPN_SEGMENTS;
    if (seg_w < 1) return fail(c, OPE_B200_E_INVALID, "fixed-pattern noise determination needs at least 8 A-scans");
    if (num_ascans < required)
        return fail(c, OPE_B200_E_INVALID, "buffer holds fewer A-scans than fpnBscanCount * ascansPerBscan");
    OPE_CU(c, cudaSetDevice(c->device));
    double* scratch = nullptr;
    OPE_CU(c, noalloc_scratch(&scratch));
    if (c->tables_dirty) {
        int rc = rebuild_tables(c);
        if (rc != OPE_B200_OK) return rc;
    }
    const long long pairs_per_seg = (seg_w + 1) / 2;
    long long gx = (pairs_per_seg + 3) / 4;
    if (gx < 1) gx = 1;
    if (gx > kNoAllocMaxGx) gx = kNoAllocMaxGx;
    const int half = c->n / 2;
    double* partial = scratch;
    double* acc = scratch + kNoAllocPartial;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ChainArgs a = make_args(c, d_in, nullptr, num_ascans, nullptr);
    // the accumulators must start at zero; the partials are fully overwritten
    OPE_CU(c, cudaMemsetAsync(acc, 0, static_cast<size_t>(FPN_SEGMENTS) * half * 3 * sizeof(double), s));
    OPE_CU(c, launch_fpn_stats(c->n, c->in_kind, c->interp, a, 0, required, seg_w, static_cast<int>(gx), partial, s));
    OPE_CU(c, launch_fpn_reduce(partial, acc, static_cast<int>(gx), half, s));
    OPE_CU(c, launch_fpn_finalize(acc, reinterpret_cast<float2*>(d_profile), half, seg_w, s));
    OPE_CU(c, cudaEventRecord(c->slot[c->active].last_use, s));
    return OPE_B200_OK;
}

}  // extern "C"
