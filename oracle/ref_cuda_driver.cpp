// Comparison driver: a C entry layer around the reference's own CUDA backend
// (ope::CudaBackend, src/backends/cuda/cuda_backend.cu + cuda_kernels.cu,
// cuFFT for the inverse DFT) compiled out of tree from the reference sources
// with the reference's default CUDA flags (--use_fast_math, sm_100). It is
// test and benchmark infrastructure: only tests and the reference arm of the
// benchmark load it, to compare against the reference's GPU path; it is not
// an oracle (cuFFT is closed) and never the product.
//
// Set-up follows Processor::Impl (src/core/processor.cpp:53-156) as the CPU
// driver does: backend->initialize(config), the output callback, then the
// generated curves, the dispersion phase handed over as interleaved float
// (cos, sin).
//
// Two ways to drive it:
//  * ope_refcuda_process: one frame, blocking (getNextAvailableInputBuffer,
//    copy in, process, wait for the output callback, copy out), for parity;
//  * ope_refcuda_fill_inputs + ope_refcuda_stream: every input IOBuffer of the
//    ring is filled once (as a frame grabber writing into the lent buffer
//    would), then frames are pushed back to back through the ring; the output
//    callback only counts frames (no consumer copy). The wall time from the
//    first buffer request to the last callback is the reference's sustained
//    end-to-end rate through its own API, host<->device copies included.
#include "backends/cuda/cuda_backend.h"
#include "processorconfiguration.h"
#include "iobuffer.h"
#include "types.h"

#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

extern "C" {

// Same layout as the CPU driver's parameter block (oracle/ref_driver.cpp).
struct ope_ref_params {
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

struct CudaRefHandle {
    ope::ProcessorConfiguration config;
    std::unique_ptr<ope::CudaBackend> backend;
    std::mutex mu;
    std::condition_variable cv;
    float* pending_out = nullptr;
    size_t out_floats = 0;
    uint64_t frames_done = 0;
    size_t in_bytes = 0;
};

thread_local std::string g_error;

int fail(const std::exception& e) {
    g_error = e.what();
    return -3;
}

bool wait_frames(CudaRefHandle* h, uint64_t target, int timeout_ms) {
    std::unique_lock<std::mutex> lk(h->mu);
    return h->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms > 0 ? timeout_ms : 600000),
                          [&] { return h->frames_done >= target; });
}

}  // namespace

extern "C" {

const char* ope_refcuda_last_error() { return g_error.c_str(); }

void* ope_refcuda_create(const ope_ref_params* p, int num_input_buffers) {
    if (!p) return nullptr;
    auto* h = new CudaRefHandle();
    try {
        h->config = make_config(*p);
        if (!h->config.validate()) throw std::invalid_argument("invalid configuration");
        h->backend = std::make_unique<ope::CudaBackend>();
        if (num_input_buffers > 0) h->backend->setNumInputBuffers(num_input_buffers);
        h->backend->initialize(h->config);
        h->backend->setOutputCallback([h](const ope::IOBuffer& out) {
            std::lock_guard<std::mutex> lk(h->mu);
            if (h->pending_out) std::memcpy(h->pending_out, out.getDataPointer(), h->out_floats * sizeof(float));
            h->frames_done++;
            h->cv.notify_all();
        });
        size_t n = static_cast<size_t>(p->signal_length);
        const float* r = h->config.getGeneratedResamplingCurve();
        h->backend->updateResamplingCurve(r, n);
        const float* w = h->config.getGeneratedWindowCurve();
        h->backend->updateWindowCurve(w, n);
        const float* ph = h->config.getGeneratedDispersionCurve();
        std::vector<float> cs(2 * n);
        for (size_t i = 0; i < n; ++i) {
            cs[2 * i] = std::cos(ph[i]);
            cs[2 * i + 1] = std::sin(ph[i]);
        }
        h->backend->updateDispersionCurve(cs.data(), cs.size());
        const auto& dp = h->config.dataParams;
        h->in_bytes = static_cast<size_t>(dp.samplesPerBuffer) * static_cast<size_t>(dp.getBytesPerSample());
        h->out_floats = static_cast<size_t>(dp.samplesPerBuffer) / 2;
    } catch (const std::exception& e) {
        g_error = e.what();
        delete h;
        return nullptr;
    }
    return h;
}

int ope_refcuda_process(void* handle, const void* input, float* output, int timeout_ms) {
    auto* h = static_cast<CudaRefHandle*>(handle);
    if (!h || !input || !output) return -1;
    uint64_t target;
    try {
        {
            std::lock_guard<std::mutex> lk(h->mu);
            h->pending_out = output;
            target = h->frames_done + 1;
        }
        ope::IOBuffer& buf = h->backend->getNextAvailableInputBuffer();
        std::memcpy(buf.getDataPointer(), input, h->in_bytes);
        h->backend->process(buf);
    } catch (const std::exception& e) {
        return fail(e);
    }
    bool ok = wait_frames(h, target, timeout_ms);
    std::lock_guard<std::mutex> lk(h->mu);
    h->pending_out = nullptr;
    return ok ? 0 : -2;
}

int ope_refcuda_request_fpn(void* handle) {
    auto* h = static_cast<CudaRefHandle*>(handle);
    if (!h) return -1;
    h->backend->requestFixedPatternNoiseDetermination();
    return 0;
}

int ope_refcuda_set_fpn(void* handle, const float* data, size_t pairs) {
    auto* h = static_cast<CudaRefHandle*>(handle);
    if (!h || !data) return -1;
    try {
        h->backend->setFixedPatternNoiseProfile(data, pairs);
    } catch (const std::exception& e) {
        return fail(e);
    }
    return 0;
}

int ope_refcuda_fill_inputs(void* handle, const void* input) {
    auto* h = static_cast<CudaRefHandle*>(handle);
    if (!h || !input) return -1;
    try {
        for (int i = 0; i < h->backend->getNumInputBuffers(); ++i)
            std::memcpy(h->backend->getInputBuffer(i).getDataPointer(), input, h->in_bytes);
    } catch (const std::exception& e) {
        return fail(e);
    }
    return 0;
}

int ope_refcuda_stream(void* handle, int frames, int timeout_ms, double* seconds) {
    auto* h = static_cast<CudaRefHandle*>(handle);
    if (!h || frames <= 0) return -1;
    uint64_t target;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->pending_out = nullptr;
        target = h->frames_done + static_cast<uint64_t>(frames);
    }
    auto t0 = std::chrono::steady_clock::now();
    try {
        for (int k = 0; k < frames; ++k) h->backend->process(h->backend->getNextAvailableInputBuffer());
    } catch (const std::exception& e) {
        return fail(e);
    }
    bool ok = wait_frames(h, target, timeout_ms);
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    return ok ? 0 : -2;
}

void ope_refcuda_destroy(void* handle) {
    auto* h = static_cast<CudaRefHandle*>(handle);
    if (!h) return;
    try {
        h->backend->cleanup();
    } catch (const std::exception&) {
    }
    h->backend.reset();
    delete h;
}

}  // extern "C"
