// ope::B200Backend over the C ABI (include/ope_b200.h).
//
// process() is asynchronous (CpuBackend::process pushes to a work queue,
// cpu_backend.cpp:473-479; CudaBackend::process enqueues, cuda_backend.cu:442-773):
// the input IOBuffer is submitted to the streaming ring and a completion thread
// (1) returns the input buffer to the free queue once its copy to the device
// has finished, (2) waits for the frame, (3) hands the frame's output IOBuffer
// to the output callback and (4) releases the ring slot after the callback
// returned -- so, unlike the reference's output ping-pong, a frame's output is
// never overwritten while a consumer reads it.
#include "b200_backend.h"

#include <condition_variable>
#include <cstdio>
#include <deque>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>

#include "../../include/ope_b200.h"

namespace ope {

namespace {

constexpr int kWaitMs = 120000;  // host-side bound on any single frame wait

ope_b200_config to_c(const ProcessorConfiguration& c, int depth, bool dc_reference_order) {
    ope_b200_config o;
    ope_b200_config_default(&o);
    o.signal_length = c.dataParams.signalLength;
    o.ascans_per_bscan = c.dataParams.ascansPerBscan;
    o.bscans_per_buffer = c.dataParams.bscansPerBuffer;
    o.input_dtype = static_cast<int32_t>(c.dataParams.inputDataType);
    o.bitshift = c.dataParams.bitshift;
    o.resampling_enabled = c.resamplingParams.enabled;
    o.interpolation = static_cast<int32_t>(c.resamplingParams.interpolationMethod);
    o.windowing_enabled = c.windowingParams.enabled;
    o.dispersion_enabled = c.dispersionParams.enabled;
    o.dc_removal_enabled = c.backgroundRemovalParams.enabled;
    o.dc_window = c.backgroundRemovalParams.rollingAverageWindowSize;
    const auto& p = c.postProcessingParams;
    o.log_scaling = p.logScaling;
    o.grayscale_min = p.grayscaleMin;
    o.grayscale_max = p.grayscaleMax;
    o.addend = p.addend;
    o.multiplicator = p.multiplicator;
    o.fpn_removal = p.fixedPatternNoiseRemoval;
    o.fpn_bscan_count = p.fixedPatternNoiseBscanCount;
    o.fpn_continuous = p.continuousFixedPatternNoiseDetermination;
    o.post_bg_removal = p.backgroundRemoval;
    o.bg_weight = p.backgroundWeight;
    o.bg_offset = p.backgroundOffset;
    o.bscan_flip = p.bscanFlip;
    o.sinusoidal_correction = p.sinusoidalScanCorrection;
    o.num_input_buffers = depth;
    o.dc_reference_order = dc_reference_order ? 1 : 0;
    return o;
}

}  // namespace

struct B200Backend::Impl {
    ope_b200_ctx* ctx = nullptr;
    ProcessorConfiguration config;
    int depth = 0;
    bool dc_reference_order = true;
    size_t in_bytes = 0, out_bytes = 0;

    std::mutex cb_mu;
    std::function<void(const IOBuffer&)> callback;

    std::vector<std::unique_ptr<IOBuffer>> inputs, outputs;

    struct Frame {
        uint64_t ticket;
        IOBuffer* in;
        bool ours;
        size_t out_idx;
    };
    std::mutex q_mu;
    std::condition_variable q_cv;
    std::deque<IOBuffer*> free_inputs;
    std::deque<Frame> pending;
    int outstanding = 0;
    uint64_t frames = 0;
    bool stop = false;
    std::thread completer;

    std::vector<float> fpn_profile, bg_profile;

    void check(int rc, const char* what) const {
        if (rc == OPE_B200_OK) return;
        std::string msg = std::string(what) + ": " + ope_b200_last_error(ctx);
        if (rc == OPE_B200_E_INVALID) throw std::invalid_argument(msg);
        throw std::runtime_error(msg);
    }

    void complete_loop() {
        while (true) {
            Frame f;
            {
                std::unique_lock<std::mutex> lk(q_mu);
                q_cv.wait(lk, [&] { return stop || !pending.empty(); });
                if (pending.empty()) return;  // stopped and drained
                f = pending.front();
                pending.pop_front();
            }
            int rc = ope_b200_input_released(ctx, f.ticket, kWaitMs);
            if (f.ours) {
                std::lock_guard<std::mutex> lk(q_mu);
                free_inputs.push_back(f.in);
            }
            q_cv.notify_all();
            const float* out = nullptr;
            if (rc == OPE_B200_OK) rc = ope_b200_wait(ctx, f.ticket, kWaitMs, &out);
            if (rc == OPE_B200_OK) {
                std::function<void(const IOBuffer&)> cb;
                {
                    std::lock_guard<std::mutex> lk(cb_mu);
                    cb = callback;
                }
                if (cb) cb(*outputs[f.out_idx]);
            } else {
                std::fprintf(stderr, "ope::B200Backend: frame %llu failed: %s\n",
                             static_cast<unsigned long long>(f.ticket), ope_b200_last_error(ctx));
                ope_b200_wait(ctx, f.ticket, kWaitMs, &out);  // make sure the slot is idle
            }
            ope_b200_release(ctx, f.ticket);
            {
                std::lock_guard<std::mutex> lk(q_mu);
                --outstanding;
            }
            q_cv.notify_all();
        }
    }

    void free_buffers() {
        for (auto* v : {&inputs, &outputs})
            for (auto& b : *v) {
                if (b && b->getDataPointer()) ope_b200_host_unregister(b->getDataPointer());
                b.reset();
            }
        inputs.clear();
        outputs.clear();
        free_inputs.clear();
    }
};

B200Backend::B200Backend() : impl(std::make_unique<Impl>()) {}

B200Backend::~B200Backend() { cleanup(); }

void B200Backend::setRollingAverageReferenceOrder(bool on) { impl->dc_reference_order = on; }

void B200Backend::initialize(const ProcessorConfiguration& config) {
    cleanup();
    auto& m = *impl;
    m.config = config;
    int nb = config.processingParams.nBuffers;
    m.depth = nb < 2 ? 2 : (nb > 4 ? 4 : nb);
    const ope_b200_config c = to_c(config, m.depth, m.dc_reference_order);
    m.check(ope_b200_create(&c, &m.ctx), "B200 backend initialization");
    const size_t samples = static_cast<size_t>(config.dataParams.signalLength) * config.dataParams.ascansPerBscan *
                           config.dataParams.bscansPerBuffer;
    m.in_bytes = samples * static_cast<size_t>(config.dataParams.getBytesPerSample());
    m.out_bytes = (samples / 2) * sizeof(float);
    for (int i = 0; i < m.depth; ++i) {
        auto in = std::make_unique<IOBuffer>();
        auto out = std::make_unique<IOBuffer>();
        if (!in->allocateMemory(m.in_bytes) || !out->allocateMemory(m.out_bytes))
            throw std::runtime_error("Failed to allocate input/output buffers");
        in->setDataType(config.dataParams.inputDataType);
        out->setDataType(DataType::FLOAT32);
        // page-locked so the ring's copies are asynchronous
        ope_b200_host_register(in->getDataPointer(), m.in_bytes);
        ope_b200_host_register(out->getDataPointer(), m.out_bytes);
        m.free_inputs.push_back(in.get());
        m.inputs.push_back(std::move(in));
        m.outputs.push_back(std::move(out));
    }
    m.stop = false;
    m.completer = std::thread([this] { impl->complete_loop(); });
}

void B200Backend::cleanup() {
    auto& m = *impl;
    {
        std::lock_guard<std::mutex> lk(m.q_mu);
        m.stop = true;
    }
    m.q_cv.notify_all();
    if (m.completer.joinable()) m.completer.join();
    if (m.ctx) {
        ope_b200_synchronize(m.ctx, nullptr);
        ope_b200_destroy(m.ctx);
        m.ctx = nullptr;
    }
    m.free_buffers();
    m.pending.clear();
    m.outstanding = 0;
    m.frames = 0;
}

void B200Backend::setOutputCallback(std::function<void(const IOBuffer&)> callback) {
    std::lock_guard<std::mutex> lk(impl->cb_mu);
    impl->callback = std::move(callback);
}

void B200Backend::process(IOBuffer& input) {
    auto& m = *impl;
    if (!m.ctx) throw std::runtime_error("B200 backend is not initialized");
    if (input.getSizeInBytes() < m.in_bytes)
        throw std::invalid_argument("Input buffer smaller than one configured buffer");
    std::unique_lock<std::mutex> lk(m.q_mu);
    m.q_cv.wait(lk, [&] { return m.stop || m.outstanding < m.depth; });
    if (m.stop) throw std::runtime_error("B200 backend is stopping");
    const size_t out_idx = m.frames % static_cast<size_t>(m.depth);
    uint64_t ticket = 0;
    m.check(ope_b200_submit_to(m.ctx, input.getDataPointer(),
                               static_cast<float*>(m.outputs[out_idx]->getDataPointer()), &ticket),
            "process");
    ++m.frames;
    ++m.outstanding;
    bool ours = false;
    for (auto& b : m.inputs) ours = ours || b.get() == &input;
    m.pending.push_back({ticket, &input, ours, out_idx});
    lk.unlock();
    m.q_cv.notify_all();
}

void B200Backend::updateConfig(const ProcessorConfiguration& config) {
    auto& m = *impl;
    m.config = config;
    if (!m.ctx) return;
    const ope_b200_config c = to_c(config, m.depth, m.dc_reference_order);
    m.check(ope_b200_update_config(m.ctx, &c), "updateConfig");
}

void B200Backend::updateResamplingCurve(const float* curve, size_t length) {
    if (!curve && length > 0) throw std::runtime_error("Invalid resampling curve pointer");
    impl->check(ope_b200_set_resampling_curve(impl->ctx, curve, length), "updateResamplingCurve");
}

void B200Backend::updateDispersionCurve(const float* curve, size_t length) {
    impl->check(ope_b200_set_dispersion_curve(impl->ctx, curve, length), "updateDispersionCurve");
}

void B200Backend::updateWindowCurve(const float* curve, size_t length) {
    if (!curve && length > 0) throw std::runtime_error("Invalid window curve pointer");
    impl->check(ope_b200_set_window_curve(impl->ctx, curve, length), "updateWindowCurve");
}

IOBuffer& B200Backend::getInputBuffer(int index) {
    if (index < 0 || index >= static_cast<int>(impl->inputs.size()))
        throw std::runtime_error("Buffer index out of range");
    return *impl->inputs[index];
}

IOBuffer& B200Backend::getNextAvailableInputBuffer() {
    auto& m = *impl;
    std::unique_lock<std::mutex> lk(m.q_mu);
    m.q_cv.wait(lk, [&] { return !m.free_inputs.empty() || m.inputs.empty(); });
    if (m.inputs.empty()) throw std::runtime_error("B200 backend is not initialized");
    IOBuffer* b = m.free_inputs.front();
    m.free_inputs.pop_front();
    return *b;
}

int B200Backend::getNumInputBuffers() const { return static_cast<int>(impl->inputs.size()); }

void B200Backend::requestPostProcessBackgroundRecording() {
    impl->check(ope_b200_request_bg_recording(impl->ctx), "requestPostProcessBackgroundRecording");
}

void B200Backend::setPostProcessBackgroundProfile(const float* background, size_t length) {
    if (!background) throw std::invalid_argument("Background curve data is null");
    impl->check(ope_b200_set_bg_profile(impl->ctx, background, length), "setPostProcessBackgroundProfile");
}

const std::vector<float>& B200Backend::getPostProcessBackgroundProfile() const {
    auto& m = *impl;
    m.bg_profile.clear();
    size_t n = 0;
    if (m.ctx && ope_b200_get_bg_profile(m.ctx, nullptr, 0, &n) == OPE_B200_OK && n) {
        m.bg_profile.resize(n);
        ope_b200_get_bg_profile(m.ctx, m.bg_profile.data(), n, &n);
    }
    return m.bg_profile;
}

void B200Backend::requestFixedPatternNoiseDetermination() {
    impl->check(ope_b200_request_fpn_determination(impl->ctx), "requestFixedPatternNoiseDetermination");
}

void B200Backend::setFixedPatternNoiseProfile(const float* profile, size_t pairs) {
    if (!profile && pairs > 0) throw std::invalid_argument("Invalid fixed-pattern noise profile pointer");
    impl->check(ope_b200_set_fpn_profile(impl->ctx, profile, pairs), "setFixedPatternNoiseProfile");
}

const std::vector<float>& B200Backend::getFixedPatternNoiseProfile() const {
    auto& m = *impl;
    m.fpn_profile.clear();
    size_t pairs = 0;
    if (m.ctx && ope_b200_get_fpn_profile(m.ctx, nullptr, 0, &pairs) == OPE_B200_OK && pairs) {
        m.fpn_profile.resize(2 * pairs);
        ope_b200_get_fpn_profile(m.ctx, m.fpn_profile.data(), pairs, &pairs);
    }
    return m.fpn_profile;
}

// Low-level per-operation API (processor.h:165-282): each operation is one
// GPU kernel of the C ABI (ope_b200_op_*, octproengine_b200/csrc/ops.cu) on
// host arrays. The reference CPU backend implements convertInput,
// kLinearization, windowing, dispersionCompensation, ifft,
// getMinimumVarianceMean and fixedPatternNoiseRemoval and returns zero vectors
// for the others; the reference CUDA backend returns empty vectors for all.
namespace {

std::vector<float> op_result(int rc, std::vector<float>&& out, const char* what) {
    if (rc != OPE_B200_OK) throw std::runtime_error(std::string(what) + ": low-level operation failed");
    return std::move(out);
}

}  // namespace

std::vector<float> B200Backend::convertInput(const void* input, IOBuffer::DataType, int bitDepth, int samples,
                                             bool) {
    std::vector<float> out(samples > 0 ? samples : 0);
    if (!input || samples <= 0) return out;
    return op_result(ope_b200_op_convert_input(input, bitDepth, samples, out.data()), std::move(out), "convertInput");
}

std::vector<float> B200Backend::rollingAverageBackgroundRemoval(const float* input, int windowSize, int lineWidth,
                                                                int numLines) {
    std::vector<float> out(static_cast<size_t>(lineWidth) * numLines);
    return op_result(ope_b200_op_rolling_dc_removal(input, windowSize, lineWidth, numLines, out.data()),
                     std::move(out), "rollingAverageBackgroundRemoval");
}

std::vector<float> B200Backend::kLinearization(const float* input, const float* resampleCurve,
                                               InterpolationMethod method, int lineWidth, int samples) {
    std::vector<float> out(samples);
    return op_result(ope_b200_op_klinearization(input, resampleCurve, static_cast<int>(method), lineWidth, samples,
                                                out.data()),
                     std::move(out), "kLinearization");
}

std::vector<float> B200Backend::windowing(const float* input, const float* windowCurve, int lineWidth, int samples) {
    std::vector<float> out(samples);
    return op_result(ope_b200_op_window_dispersion(input, windowCurve, nullptr, 1, lineWidth, samples, out.data()),
                     std::move(out), "windowing");
}

std::vector<float> B200Backend::dispersionCompensation(const float* input, const float* phaseComplex, int lineWidth,
                                                       int samples) {
    std::vector<float> out(samples);
    return op_result(ope_b200_op_window_dispersion(input, nullptr, phaseComplex, 2, lineWidth, samples, out.data()),
                     std::move(out), "dispersionCompensation");
}

std::vector<float> B200Backend::kLinearizationAndWindowing(const float* input, const float* resampleCurve,
                                                           const float* windowCurve, InterpolationMethod method,
                                                           int lineWidth, int samples) {
    std::vector<float> k = kLinearization(input, resampleCurve, method, lineWidth, lineWidth);
    return windowing(k.data(), windowCurve, lineWidth, samples);
}

std::vector<float> B200Backend::kLinearizationAndWindowingAndDispersion(const float* input, const float* resampleCurve,
                                                                        const float* windowCurve,
                                                                        const float* phaseComplex,
                                                                        InterpolationMethod method, int lineWidth,
                                                                        int samples) {
    std::vector<float> k = kLinearizationAndWindowing(input, resampleCurve, windowCurve, method, lineWidth, lineWidth);
    return dispersionCompensation(k.data(), phaseComplex, lineWidth, samples);
}

std::vector<float> B200Backend::dispersionCompensationAndWindowing(const float* input, const float* phaseComplex,
                                                                   const float* windowCurve, int lineWidth,
                                                                   int samples) {
    std::vector<float> out(samples);
    return op_result(ope_b200_op_window_dispersion(input, windowCurve, phaseComplex, 3, lineWidth, samples,
                                                   out.data()),
                     std::move(out), "dispersionCompensationAndWindowing");
}

std::vector<float> B200Backend::fft(const float* input, int lineWidth, int) {
    std::vector<float> out(lineWidth);
    return op_result(ope_b200_op_dft_magnitude(input, lineWidth, 0, out.data()), std::move(out), "fft");
}

std::vector<float> B200Backend::ifft(const float* input, int lineWidth, int) {
    std::vector<float> out(lineWidth);
    return op_result(ope_b200_op_dft_magnitude(input, lineWidth, 1, out.data()), std::move(out), "ifft");
}

std::vector<float> B200Backend::getMinimumVarianceMean(const float* input, int width, int height, int segments) {
    if (!input) return {};
    std::vector<float> out(static_cast<size_t>(width) * 2);
    return op_result(ope_b200_op_min_variance_mean(input, width, height, segments, out.data()), std::move(out),
                     "getMinimumVarianceMean");
}

std::vector<float> B200Backend::fixedPatternNoiseRemoval(const float* input, const float* meanALine, int lineWidth,
                                                         int numLines) {
    if (!input) return {};
    std::vector<float> out(static_cast<size_t>(lineWidth) * numLines);
    return op_result(ope_b200_op_fpn_removal(input, meanALine, lineWidth, numLines, out.data()), std::move(out),
                     "fixedPatternNoiseRemoval");
}

std::vector<float> B200Backend::postProcessTruncate(const float* input, bool logScaling, float grayscaleMax,
                                                    float grayscaleMin, float addend, float multiplicator,
                                                    int lineWidth, int samples) {
    const long long lines = lineWidth > 1 ? (2LL * samples) / lineWidth : 0;
    std::vector<float> out(static_cast<size_t>(lines) * (lineWidth / 2));
    if (lines == 0) return out;
    return op_result(ope_b200_op_truncate(input, logScaling ? 1 : 0, grayscaleMax, grayscaleMin, addend, multiplicator,
                                          lineWidth, lines, out.data()),
                     std::move(out), "postProcessTruncate");
}

std::vector<float> B200Backend::bscanFlip(const float* input, int lineWidth, int linesPerBscan, int numBscans) {
    std::vector<float> out(static_cast<size_t>(lineWidth) * linesPerBscan * numBscans);
    return op_result(ope_b200_op_bscan_flip(input, lineWidth, linesPerBscan, numBscans, out.data()), std::move(out),
                     "bscanFlip");
}

std::vector<float> B200Backend::sinusoidalScanCorrection(const float* input, const float* resampleCurve,
                                                         int lineWidth, int linesPerBscan, int numBscans) {
    std::vector<float> out(static_cast<size_t>(lineWidth) * linesPerBscan * numBscans);
    return op_result(ope_b200_op_sinusoidal_correction(input, resampleCurve, lineWidth, linesPerBscan, numBscans,
                                                       out.data()),
                     std::move(out), "sinusoidalScanCorrection");
}

std::vector<float> B200Backend::postProcessBackgroundSubtraction(const float* input, const float* backgroundLine,
                                                                 float weight, float offset, int lineWidth,
                                                                 int samples) {
    std::vector<float> out(samples);
    return op_result(ope_b200_op_background_subtraction(input, backgroundLine, weight, offset, lineWidth, samples,
                                                        out.data()),
                     std::move(out), "postProcessBackgroundSubtraction");
}

}  // namespace ope
