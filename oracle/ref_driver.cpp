// Test-oracle driver: a C entry layer around the reference's own CPU backend
// (ope::CpuBackend, src/backends/cpu/cpu_backend.cpp) compiled out of tree from
// the reference sources. It is test infrastructure: only tests, the smoke check
// and the CPU-baseline leg of the benchmark load it, and never as the product.
//
// What it reproduces from the reference, in code of its own:
//  * curve hand-off as Processor::Impl does it (src/core/processor.cpp:53-99):
//    generated or custom resampling / window curves, and the dispersion phase
//    converted to interleaved (cos, sin) pairs with float std::cos/std::sin;
//  * the setup order of Processor::Impl::initialize (processor.cpp:135-156):
//    backend->initialize(config), callback installation, then curves;
//  * one blocking "process a frame" call: getNextAvailableInputBuffer, copy in,
//    process, wait for the output callback, copy out (processor.cpp:348-365).
#include "backends/cpu/cpu_backend.h"
#include "backends/cpu/cpu_kernels.h"
#include "processorconfiguration.h"
#include "iobuffer.h"
#include "types.h"

#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

extern "C" {

struct ope_ref_params {
    int signal_length;
    int ascans_per_bscan;
    int bscans_per_buffer;
    int input_dtype;  // ope::DataType numeric value
    int resampling_enabled;
    int interpolation;  // ope::InterpolationMethod
    float resampling_coeffs[4];
    int windowing_enabled;
    int window_type;  // ope::WindowType
    float window_center;
    float window_fill;
    int dispersion_enabled;
    float dispersion_coeffs[4];
    float dispersion_factor;
    int dc_removal_enabled;
    int dc_window;
    int log_scaling;
    float grayscale_min;
    float grayscale_max;
    float addend;
    float multiplicator;
    int fpn_removal;
    int fpn_bscan_count;
    int fpn_continuous;
    int post_bg_removal;
    float bg_weight;
    float bg_offset;
};

}  // extern "C"

namespace {

ope::ProcessorConfiguration make_config(const ope_ref_params& p) {
    ope::ProcessorConfiguration c;
    c.dataParams.signalLength = p.signal_length;
    c.dataParams.ascansPerBscan = p.ascans_per_bscan;
    c.dataParams.bscansPerBuffer = p.bscans_per_buffer;
    c.dataParams.samplesPerBuffer = p.signal_length * p.ascans_per_bscan * p.bscans_per_buffer;
    c.dataParams.inputDataType = static_cast<ope::DataType>(p.input_dtype);
    c.resamplingParams.enabled = p.resampling_enabled != 0;
    c.resamplingParams.interpolationMethod = static_cast<ope::InterpolationMethod>(p.interpolation);
    for (int i = 0; i < 4; ++i) c.resamplingParams.coefficients[i] = p.resampling_coeffs[i];
    c.windowingParams.enabled = p.windowing_enabled != 0;
    c.windowingParams.windowType = static_cast<ope::WindowType>(p.window_type);
    c.windowingParams.windowCenterPosition = p.window_center;
    c.windowingParams.windowFillFactor = p.window_fill;
    c.dispersionParams.enabled = p.dispersion_enabled != 0;
    for (int i = 0; i < 4; ++i) c.dispersionParams.coefficients[i] = p.dispersion_coeffs[i];
    c.dispersionParams.factor = p.dispersion_factor;
    c.backgroundRemovalParams.enabled = p.dc_removal_enabled != 0;
    c.backgroundRemovalParams.rollingAverageWindowSize = p.dc_window;
    c.postProcessingParams.logScaling = p.log_scaling != 0;
    c.postProcessingParams.grayscaleMin = p.grayscale_min;
    c.postProcessingParams.grayscaleMax = p.grayscale_max;
    c.postProcessingParams.addend = p.addend;
    c.postProcessingParams.multiplicator = p.multiplicator;
    c.postProcessingParams.fixedPatternNoiseRemoval = p.fpn_removal != 0;
    c.postProcessingParams.fixedPatternNoiseBscanCount = p.fpn_bscan_count;
    c.postProcessingParams.continuousFixedPatternNoiseDetermination = p.fpn_continuous != 0;
    c.postProcessingParams.backgroundRemoval = p.post_bg_removal != 0;
    c.postProcessingParams.backgroundWeight = p.bg_weight;
    c.postProcessingParams.backgroundOffset = p.bg_offset;
    return c;
}

// Phase -> interleaved (cos, sin), float overloads, as processor.cpp:92-97.
std::vector<float> phase_to_cos_sin(const float* phase, size_t n) {
    std::vector<float> out(2 * n);
    for (size_t i = 0; i < n; ++i) {
        float ph = phase[i];
        out[2 * i] = std::cos(ph);
        out[2 * i + 1] = std::sin(ph);
    }
    return out;
}

struct RefHandle {
    ope_ref_params params;
    ope::ProcessorConfiguration config;
    std::unique_ptr<ope::CpuBackend> backend;
    std::mutex mu;
    std::condition_variable cv;
    float* pending_out = nullptr;
    size_t out_floats = 0;
    uint64_t frames_done = 0;
    std::string error;
};

}  // namespace

extern "C" {

int ope_ref_generate_curves(const ope_ref_params* p, float* resample, float* window, float* phase,
                            float* cos_sin) {
    if (!p || p->signal_length <= 0) return -1;
    ope::ProcessorConfiguration c = make_config(*p);
    size_t n = static_cast<size_t>(p->signal_length);
    const float* r = c.getGeneratedResamplingCurve();
    if (resample) std::memcpy(resample, r, n * sizeof(float));
    const float* w = c.getGeneratedWindowCurve();
    if (window) std::memcpy(window, w, n * sizeof(float));
    const float* ph = c.getGeneratedDispersionCurve();
    if (phase) std::memcpy(phase, ph, n * sizeof(float));
    if (cos_sin) {
        std::vector<float> cs = phase_to_cos_sin(ph, n);
        std::memcpy(cos_sin, cs.data(), cs.size() * sizeof(float));
    }
    return 0;
}

void* ope_ref_create(const ope_ref_params* p) {
    if (!p) return nullptr;
    auto* h = new RefHandle();
    h->params = *p;
    h->config = make_config(*p);
    if (!h->config.validate()) {
        delete h;
        return nullptr;
    }
    h->backend = std::make_unique<ope::CpuBackend>();
    h->backend->initialize(h->config);
    h->backend->setOutputCallback([h](const ope::IOBuffer& out) {
        std::lock_guard<std::mutex> lk(h->mu);
        if (h->pending_out) {
            std::memcpy(h->pending_out, out.getDataPointer(), h->out_floats * sizeof(float));
        }
        h->frames_done++;
        h->cv.notify_all();
    });
    size_t n = static_cast<size_t>(p->signal_length);
    std::vector<float> r(h->config.getGeneratedResamplingCurve(), h->config.getGeneratedResamplingCurve() + n);
    h->backend->updateResamplingCurve(r.data(), r.size());
    std::vector<float> w(h->config.getGeneratedWindowCurve(), h->config.getGeneratedWindowCurve() + n);
    h->backend->updateWindowCurve(w.data(), w.size());
    std::vector<float> cs = phase_to_cos_sin(h->config.getGeneratedDispersionCurve(), n);
    h->backend->updateDispersionCurve(cs.data(), cs.size());
    return h;
}

// kind: 0 resampling curve (n floats), 1 window curve (n floats),
//       2 dispersion phase (n floats, converted to cos/sin like the Processor),
//       3 dispersion cos/sin interleaved (2n floats, passed as is).
int ope_ref_set_curve(void* handle, int kind, const float* data, size_t n) {
    auto* h = static_cast<RefHandle*>(handle);
    if (!h || !data) return -1;
    switch (kind) {
        case 0: h->backend->updateResamplingCurve(data, n); break;
        case 1: h->backend->updateWindowCurve(data, n); break;
        case 2: {
            std::vector<float> cs = phase_to_cos_sin(data, n);
            h->backend->updateDispersionCurve(cs.data(), cs.size());
            break;
        }
        case 3: h->backend->updateDispersionCurve(data, n); break;
        default: return -1;
    }
    return 0;
}

int ope_ref_process(void* handle, const void* input, float* output, int timeout_ms) {
    auto* h = static_cast<RefHandle*>(handle);
    if (!h || !input || !output) return -1;
    const auto& dp = h->config.dataParams;
    size_t in_bytes = static_cast<size_t>(dp.samplesPerBuffer) * static_cast<size_t>(dp.getBytesPerSample());
    size_t out_floats = static_cast<size_t>(dp.samplesPerBuffer) / 2;
    uint64_t target;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->pending_out = output;
        h->out_floats = out_floats;
        target = h->frames_done + 1;
    }
    ope::IOBuffer& buf = h->backend->getNextAvailableInputBuffer();
    std::memcpy(buf.getDataPointer(), input, in_bytes);
    h->backend->process(buf);
    std::unique_lock<std::mutex> lk(h->mu);
    bool ok = h->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms > 0 ? timeout_ms : 600000),
                             [&] { return h->frames_done >= target; });
    h->pending_out = nullptr;
    return ok ? 0 : -2;
}

void ope_ref_update_params(void* handle, const ope_ref_params* p) {
    auto* h = static_cast<RefHandle*>(handle);
    if (!h || !p) return;
    h->params = *p;
    h->config = make_config(*p);
    h->backend->updateConfig(h->config);
}

void ope_ref_request_fpn(void* handle) {
    auto* h = static_cast<RefHandle*>(handle);
    if (h) h->backend->requestFixedPatternNoiseDetermination();
}

int ope_ref_get_fpn(void* handle, float* out, size_t cap_floats) {
    auto* h = static_cast<RefHandle*>(handle);
    if (!h) return -1;
    const std::vector<float>& v = h->backend->getFixedPatternNoiseProfile();
    size_t n = v.size() < cap_floats ? v.size() : cap_floats;
    if (out && n) std::memcpy(out, v.data(), n * sizeof(float));
    return static_cast<int>(v.size());
}

void ope_ref_set_fpn(void* handle, const float* data, size_t pairs) {
    auto* h = static_cast<RefHandle*>(handle);
    if (h) h->backend->setFixedPatternNoiseProfile(data, pairs);
}

void ope_ref_request_bg(void* handle) {
    auto* h = static_cast<RefHandle*>(handle);
    if (h) h->backend->requestPostProcessBackgroundRecording();
}

int ope_ref_get_bg(void* handle, float* out, size_t cap) {
    auto* h = static_cast<RefHandle*>(handle);
    if (!h) return -1;
    const std::vector<float>& v = h->backend->getPostProcessBackgroundProfile();
    size_t n = v.size() < cap ? v.size() : cap;
    if (out && n) std::memcpy(out, v.data(), n * sizeof(float));
    return static_cast<int>(v.size());
}

int ope_ref_set_bg(void* handle, const float* data, size_t n) {
    auto* h = static_cast<RefHandle*>(handle);
    if (!h) return -1;
    try {
        h->backend->setPostProcessBackgroundProfile(data, n);
    } catch (...) {
        return -1;
    }
    return 0;
}

void ope_ref_destroy(void* handle) {
    auto* h = static_cast<RefHandle*>(handle);
    if (!h) return;
    h->backend->cleanup();
    h->backend.reset();
    delete h;
}

// ---- low-level operations of the reference CPU backend (processor.h:165-282) ----

static ope::CpuBackend* lowlevel_backend(int n) {
    // The CPU low-level ops need an initialized backend only for ifft (plan).
    thread_local std::unique_ptr<ope::CpuBackend> be;
    thread_local int be_n = 0;
    if (!be || be_n != n) {
        if (be) be->cleanup();
        be = std::make_unique<ope::CpuBackend>();
        ope::ProcessorConfiguration c;
        c.dataParams.signalLength = n;
        c.dataParams.ascansPerBscan = 1;
        c.dataParams.bscansPerBuffer = 1;
        c.dataParams.samplesPerBuffer = n;
        be->initialize(c);
        be_n = n;
    }
    return be.get();
}

int ope_ref_convert_input(const void* in, int dtype, int samples, float* out) {
    ope::CpuBackend* be = lowlevel_backend(samples > 0 ? samples : 1);
    ope::DataType t = static_cast<ope::DataType>(dtype);
    std::vector<float> v = be->convertInput(in, t, ope::getDataTypeBitDepth(t), samples, false);
    std::memcpy(out, v.data(), v.size() * sizeof(float));
    return 0;
}

int ope_ref_klinearization(const float* in, const float* curve, int method, int n, float* out) {
    ope::CpuBackend* be = lowlevel_backend(n);
    std::vector<float> v = be->kLinearization(in, curve, static_cast<ope::InterpolationMethod>(method), n, n);
    std::memcpy(out, v.data(), v.size() * sizeof(float));
    return 0;
}

int ope_ref_windowing(const float* in, const float* win, int n, float* out) {
    ope::CpuBackend* be = lowlevel_backend(n);
    std::vector<float> v = be->windowing(in, win, n, n);
    std::memcpy(out, v.data(), v.size() * sizeof(float));
    return 0;
}

int ope_ref_min_var_mean(const float* in, int width, int height, int segments, float* out) {
    ope::CpuBackend* be = lowlevel_backend(width);
    std::vector<float> v = be->getMinimumVarianceMean(in, width, height, segments);
    std::memcpy(out, v.data(), v.size() * sizeof(float));
    return static_cast<int>(v.size());
}

int ope_ref_ifft_magnitude(const float* in, int n, float* out) {
    ope::CpuBackend* be = lowlevel_backend(n);
    std::vector<float> v = be->ifft(in, n, n);
    std::memcpy(out, v.data(), v.size() * sizeof(float));
    return 0;
}

// The reference's rolling-average DC removal of one line (its float prefix
// sum; the CpuBackend's low-level rollingAverageBackgroundRemoval does not run it).
int ope_ref_rolling_dc(const float* in, int n, int window, float* out) {
    std::vector<std::complex<float>> v(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) v[i] = std::complex<float>(in[i], 0.0f);
    ope::cpu_kernels::rollingAverageDCRemoval(v, static_cast<size_t>(window));
    for (int i = 0; i < n; ++i) out[i] = v[i].real();
    return 0;
}

int ope_ref_fft_shim_precision(int mode) {
    ope_fftw_shim_set_precision(mode);
    return ope_fftw_shim_get_precision();
}

}  // extern "C"
