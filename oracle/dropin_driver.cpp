// Drop-in check driver: a C entry layer around the reference's OWN
// ope::Processor (src/core/processor.cpp, built out of tree with the
// Backend::B200 patch applied to a copy, see dropin_patch.py), so a test can
// run the same frame through Backend::CPU and Backend::B200 of one reference
// library and compare them, as the reference's own comparison test does for
// CPU and CUDA (tests/test_backend_output_comparison.cpp:18-45). TEST
// INFRASTRUCTURE ONLY: nothing of the product links it.
//
// Every step goes through the reference's public API: setConfig, the output
// callback, initialize, getNextAvailableInputBuffer, process, and the
// fixed-pattern-noise calls.
#include "processor.h"
#include "processorconfiguration.h"
#include "iobuffer.h"
#include "types.h"

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <string>

extern "C" {

// the same parameter block as ref_driver.cpp
struct ope_dropin_params {
    int signal_length;
    int ascans_per_bscan;
    int bscans_per_buffer;
    int input_dtype;
    int resampling_enabled;
    int interpolation;
    float resampling_coeffs[4];
    int windowing_enabled;
    int window_type;
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

void ope_fftw_shim_set_precision(int mode);

}  // extern "C"

namespace {

thread_local std::string t_error;

ope::ProcessorConfiguration make_config(const ope_dropin_params& p) {
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

struct Handle {
    std::unique_ptr<ope::Processor> proc;
    size_t in_bytes = 0, out_floats = 0;
    std::mutex mu;
    std::condition_variable cv;
    float* pending_out = nullptr;
    uint64_t frames_done = 0;
};

}  // namespace

extern "C" {

__attribute__((visibility("default"))) const char* ope_dropin_last_error() { return t_error.c_str(); }

// backend: the numeric ope::Backend value (CUDA 0, CPU 1, B200 2 in the patched library)
__attribute__((visibility("default"))) void* ope_dropin_create(int backend, const ope_dropin_params* p) {
    if (!p) return nullptr;
    try {
        auto h = std::make_unique<Handle>();
        h->proc = std::make_unique<ope::Processor>(static_cast<ope::Backend>(backend));
        const ope::ProcessorConfiguration c = make_config(*p);
        h->proc->setConfig(c);
        Handle* raw = h.get();
        h->proc->setOutputCallback([raw](const ope::IOBuffer& out) {
            std::lock_guard<std::mutex> lk(raw->mu);
            if (raw->pending_out)
                std::memcpy(raw->pending_out, out.getDataPointer(), raw->out_floats * sizeof(float));
            raw->frames_done++;
            raw->cv.notify_all();
        });
        h->proc->initialize();
        h->in_bytes = static_cast<size_t>(c.dataParams.samplesPerBuffer) * c.dataParams.getBytesPerSample();
        h->out_floats = static_cast<size_t>(c.dataParams.samplesPerBuffer) / 2;
        return h.release();
    } catch (const std::exception& e) {
        t_error = e.what();
        return nullptr;
    }
}

// One frame: next available input buffer, copy in, process, wait for the
// output callback (bounded), copy out. 0 on success, -1 on an exception, -2
// on a timeout.
__attribute__((visibility("default"))) int ope_dropin_process(void* handle, const void* input, float* output,
                                                             int timeout_ms) {
    auto* h = static_cast<Handle*>(handle);
    if (!h || !input || !output) return -1;
    try {
        ope::IOBuffer& buf = h->proc->getNextAvailableInputBuffer();
        std::memcpy(buf.getDataPointer(), input, h->in_bytes);
        uint64_t target;
        {
            std::lock_guard<std::mutex> lk(h->mu);
            h->pending_out = output;
            target = h->frames_done + 1;
        }
        h->proc->process(buf);
        std::unique_lock<std::mutex> lk(h->mu);
        const bool ok = h->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                       [&] { return h->frames_done >= target; });
        h->pending_out = nullptr;
        if (!ok) {
            t_error = "timed out waiting for the output callback";
            return -2;
        }
        return 0;
    } catch (const std::exception& e) {
        t_error = e.what();
        return -1;
    }
}

__attribute__((visibility("default"))) int ope_dropin_request_fpn(void* handle) {
    auto* h = static_cast<Handle*>(handle);
    if (!h) return -1;
    h->proc->requestFixedPatternNoiseDetermination();
    return 0;
}

__attribute__((visibility("default"))) int ope_dropin_set_fpn(void* handle, const float* data, size_t pairs) {
    auto* h = static_cast<Handle*>(handle);
    if (!h || !data) return -1;
    try {
        h->proc->setFixedPatternNoiseProfile(data, pairs);
        return 0;
    } catch (const std::exception& e) {
        t_error = e.what();
        return -1;
    }
}

// Copies the processor's FPN profile (interleaved floats); returns the float
// count (getFixedPatternNoiseProfileSize counts complex pairs).
__attribute__((visibility("default"))) long long ope_dropin_get_fpn(void* handle, float* out, size_t cap_floats) {
    auto* h = static_cast<Handle*>(handle);
    if (!h || !h->proc->hasFixedPatternNoiseProfile()) return 0;
    const size_t n = 2 * h->proc->getFixedPatternNoiseProfileSize();
    if (out) std::memcpy(out, h->proc->getFixedPatternNoiseProfile(), (n < cap_floats ? n : cap_floats) * sizeof(float));
    return static_cast<long long>(n);
}

__attribute__((visibility("default"))) int ope_dropin_backend(void* handle) {
    auto* h = static_cast<Handle*>(handle);
    return h ? static_cast<int>(h->proc->getBackend()) : -1;
}

__attribute__((visibility("default"))) void ope_dropin_fft_precision(int mode) { ope_fftw_shim_set_precision(mode); }

__attribute__((visibility("default"))) void ope_dropin_destroy(void* handle) { delete static_cast<Handle*>(handle); }

}  // extern "C"
