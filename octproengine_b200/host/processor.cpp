// ope::Processor over the B200 backend: the facade of the reference's
// src/core/processor.cpp (lifecycle, hot-swap setters, curve selection,
// profile persistence) driving B200Backend through the ProcessingBackend seam.
//
// One difference in behaviour: the reference's simple setters
// (enableLogScaling, setGrayscaleRange, enableBscanFlip, ...,
// src/core/processor.cpp:522-568) only change the Processor's copy of the
// configuration, which the backends copied at initialize(), so they take
// effect only after a re-initialization. Here every setter that changes a
// processing parameter forwards the configuration with updateConfig() when
// the processor is initialized, so it takes effect from the next submitted
// buffer on.
#include "../../include/ope/processor.h"

#include <algorithm>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ope_b200.h"
#include "b200_backend.h"
#include "callback_manager.h"

namespace ope {

class Processor::Impl {
public:
    ProcessorConfiguration config;
    std::unique_ptr<ProcessingBackend> backend;
    Backend backendType;
    bool initialized = false;
    ProcessorConfiguration::DataParameters lastInit;
    CallbackManager callbacks;

    explicit Impl(Backend type) : backendType(type) { createBackend(type); }
    ~Impl() {
        if (backend && initialized) backend->cleanup();
    }

    void createBackend(Backend type) {
        // This library is the single-backend build: Backend::CPU and
        // Backend::CUDA are the OCTproEngine library's own backends, which hold
        // all three once B200Backend is added to it (the Backend::B200 patch).
        switch (type) {
            case Backend::B200:
                backend = std::make_unique<B200Backend>();
                break;
            case Backend::CPU:
            case Backend::CUDA:
                throw std::invalid_argument(
                    std::string("Backend::") + (type == Backend::CPU ? "CPU" : "CUDA") +
                    " is not in this build, which holds the B200 backend only: select Backend::B200, or build "
                    "the OCTproEngine library with the Backend::B200 patch to have all three side by side");
            default:
                throw std::runtime_error("Unknown backend type");
        }
        backendType = type;
    }

    std::vector<float> resamplingCurve() const {
        const auto& r = config.resamplingParams;
        if (r.useCustomCurve && config.hasCustomResamplingCurve())
            return {config.getCustomResamplingCurve(),
                    config.getCustomResamplingCurve() + config.getCustomResamplingCurveSize()};
        const float* g = config.getGeneratedResamplingCurve();
        return {g, g + config.getGeneratedResamplingCurveSize()};
    }

    std::vector<float> windowCurve() const {
        if (config.windowingParams.useCustomCurve && config.hasCustomWindowCurve())
            return {config.getCustomWindowCurve(), config.getCustomWindowCurve() + config.getCustomWindowCurveSize()};
        const float* g = config.getGeneratedWindowCurve();
        return {g, g + config.getGeneratedWindowCurveSize()};
    }

    // phase (custom or generated) -> interleaved cos/sin, as
    // src/core/processor.cpp:77-99 converts it for the backends
    std::vector<float> dispersionCurve() const {
        const float* ph;
        size_t n;
        if (config.dispersionParams.useCustomCurve && config.hasCustomDispersionCurve()) {
            ph = config.getCustomDispersionCurve();
            n = config.getCustomDispersionCurveSize();
        } else {
            ph = config.getGeneratedDispersionCurve();
            n = config.getGeneratedDispersionCurveSize();
        }
        std::vector<float> cs(2 * n);
        if (n) ope_b200_phase_to_cos_sin(ph, n, cs.data());
        return cs;
    }

    // A dimension change since the last initialize() is applied by the
    // re-initialization at the next buffer request or process(); until then
    // the backend still holds the old dimensions and gets no updates.
    bool live() const { return initialized && !dimsChanged(config.dataParams, lastInit); }

    void pushResampling() {
        if (!live()) return;
        auto c = resamplingCurve();
        backend->updateResamplingCurve(c.data(), c.size());
    }
    void pushWindow() {
        if (!live()) return;
        auto c = windowCurve();
        backend->updateWindowCurve(c.data(), c.size());
    }
    void pushDispersion() {
        if (!live()) return;
        auto c = dispersionCurve();
        backend->updateDispersionCurve(c.data(), c.size());
    }
    void pushCurves() {
        pushResampling();
        pushWindow();
        pushDispersion();
    }
    void pushConfig() {
        if (live()) backend->updateConfig(config);
    }

    void pushProfiles() {
        if (config.hasCustomFixedPatternNoiseProfile() &&
            config.getCustomFixedPatternNoiseProfileSize() == static_cast<size_t>(config.dataParams.signalLength / 2))
            backend->setFixedPatternNoiseProfile(config.getCustomFixedPatternNoiseProfile(),
                                                 config.getCustomFixedPatternNoiseProfileSize());
        if (config.hasCustomPostProcessBackgroundProfile())
            backend->setPostProcessBackgroundProfile(config.getCustomPostProcessBackgroundProfile(),
                                                     config.getCustomPostProcessBackgroundProfileSize());
    }

    bool dimsChanged(const ProcessorConfiguration::DataParameters& a,
                     const ProcessorConfiguration::DataParameters& b) const {
        return a.signalLength != b.signalLength || a.samplesPerBuffer != b.samplesPerBuffer ||
               a.ascansPerBscan != b.ascansPerBscan || a.bscansPerBuffer != b.bscansPerBuffer ||
               a.inputDataType != b.inputDataType;
    }

    void initialize() {
        if (!config.validate()) throw std::runtime_error("Invalid processor configuration");
        if (initialized) backend->cleanup();
        initialized = false;
        backend->initialize(config);
        backend->setOutputCallback([this](const IOBuffer& out) { callbacks.invokeAll(out); });
        initialized = true;
        lastInit = config.dataParams;
        pushCurves();
        pushProfiles();
    }

    void ensureInitialized() {
        if (!initialized || dimsChanged(config.dataParams, lastInit)) initialize();
    }

    void cleanup() {
        if (initialized) {
            backend->cleanup();
            initialized = false;
        }
    }
};

Processor::Processor(Backend backend) : impl(std::make_unique<Impl>(backend)) {}
Processor::~Processor() = default;

void Processor::initialize() { impl->ensureInitialized(); }
void Processor::cleanup() { impl->cleanup(); }
bool Processor::isInitialized() const { return impl->initialized; }

void Processor::loadConfigurationFromFile(const std::string& filepath) {
    ProcessorConfiguration c = impl->config;
    if (!c.loadFromFile(filepath)) throw std::runtime_error("Failed to load configuration from: " + filepath);
    setConfig(c);
}

void Processor::saveConfigurationToFile(const std::string& filepath) const {
    if (!impl->config.saveToFile(filepath)) throw std::runtime_error("Failed to save configuration to: " + filepath);
}

const ProcessorConfiguration& Processor::getConfig() const { return impl->config; }

void Processor::setConfig(const ProcessorConfiguration& config) {
    const bool dims = impl->dimsChanged(impl->config.dataParams, config.dataParams);
    impl->config = config;
    if (!impl->initialized) return;
    if (dims) {
        impl->initialize();
    } else {
        impl->pushConfig();
        impl->pushCurves();
    }
}

void Processor::setInputParameters(int samplesPerRawAscan, int ascansPerBscan, int bscansPerBuffer, DataType type) {
    auto& d = impl->config.dataParams;
    const int old = d.signalLength;
    d.signalLength = samplesPerRawAscan;
    d.ascansPerBscan = ascansPerBscan;
    d.bscansPerBuffer = bscansPerBuffer;
    d.samplesPerBuffer = samplesPerRawAscan * ascansPerBscan * bscansPerBuffer;
    d.inputDataType = type;
    if (samplesPerRawAscan != old) impl->config.adjustAllCustomCurves();
    // the backend picks the new dimensions up at the next initialize()/process()
}

void Processor::setBackend(Backend backend) {
    if (impl->backendType == backend) return;
    impl->cleanup();
    impl->createBackend(backend);
}

Backend Processor::getBackend() const { return impl->backendType; }

void Processor::process(IOBuffer& input) {
    impl->ensureInitialized();
    impl->backend->process(input);
}

void Processor::setOutputCallback(OutputCallback callback) {
    impl->callbacks.clear();
    impl->callbacks.addCallback(std::move(callback));
}
Processor::CallbackId Processor::addOutputCallback(OutputCallback callback) {
    return impl->callbacks.addCallback(std::move(callback));
}
bool Processor::removeOutputCallback(CallbackId id) { return impl->callbacks.removeCallback(id); }
void Processor::clearOutputCallbacks() { impl->callbacks.clear(); }
size_t Processor::getCallbackCount() const { return impl->callbacks.getCallbackCount(); }

IOBuffer& Processor::getInputBuffer(int index) {
    impl->ensureInitialized();
    return impl->backend->getInputBuffer(index);
}
int Processor::getNumInputBuffers() const { return impl->initialized ? impl->backend->getNumInputBuffers() : 0; }
IOBuffer& Processor::getNextAvailableInputBuffer() {
    impl->ensureInitialized();
    return impl->backend->getNextAvailableInputBuffer();
}

// ---- resampling -----------------------------------------------------------

void Processor::setResamplingCoefficients(const float coefficients[4]) {
    auto& r = impl->config.resamplingParams;
    std::copy(coefficients, coefficients + 4, r.coefficients);
    r.useCoefficients = true;
    r.useCustomCurve = false;
    impl->pushResampling();
}

void Processor::setCustomResamplingCurve(const float* curve, size_t length) {
    if (!curve || length == 0) throw std::invalid_argument("Invalid custom resampling curve");
    impl->config.setCustomResamplingCurve(curve, length);
    impl->config.resamplingParams.useCustomCurve = true;
    impl->config.resamplingParams.useCoefficients = false;
    impl->pushResampling();
}

void Processor::useCustomResamplingCurve(bool useCustom) {
    auto& r = impl->config.resamplingParams;
    if (useCustom && !impl->config.hasCustomResamplingCurve())
        throw std::runtime_error("No custom resampling curve set. Call setCustomResamplingCurve() first.");
    r.useCustomCurve = useCustom;
    r.useCoefficients = !useCustom;
    impl->pushResampling();
}

void Processor::enableResampling(bool enable) {
    impl->config.resamplingParams.enabled = enable;
    impl->pushConfig();
}

void Processor::setInterpolationMethod(InterpolationMethod method) {
    impl->config.resamplingParams.interpolationMethod = method;
    impl->pushConfig();
}

// ---- dispersion -----------------------------------------------------------

void Processor::setDispersionCoefficients(const float coefficients[4], float factor) {
    auto& p = impl->config.dispersionParams;
    std::copy(coefficients, coefficients + 4, p.coefficients);
    p.factor = factor;
    p.useCoefficients = true;
    p.useCustomCurve = false;
    impl->pushDispersion();
}

void Processor::setCustomDispersionCurve(const float* curve, size_t length) {
    if (!curve || length == 0) throw std::invalid_argument("Invalid custom dispersion curve");
    impl->config.setCustomDispersionCurve(curve, length);
    impl->config.dispersionParams.useCustomCurve = true;
    impl->config.dispersionParams.useCoefficients = false;
    impl->pushDispersion();
}

void Processor::useCustomDispersionCurve(bool useCustom) {
    auto& p = impl->config.dispersionParams;
    if (useCustom && !impl->config.hasCustomDispersionCurve())
        throw std::runtime_error("No custom dispersion curve set. Call setCustomDispersionCurve() first.");
    p.useCustomCurve = useCustom;
    p.useCoefficients = !useCustom;
    impl->pushDispersion();
}

void Processor::enableDispersionCompensation(bool enable) {
    impl->config.dispersionParams.enabled = enable;
    impl->pushConfig();
}

// ---- windowing ------------------------------------------------------------

void Processor::setWindowParameters(WindowType type, float centerPosition, float fillFactor) {
    auto& w = impl->config.windowingParams;
    w.windowType = type;
    w.windowCenterPosition = centerPosition;
    w.windowFillFactor = fillFactor;
    w.useCustomCurve = false;  // the custom curve is kept for later toggling
    impl->pushWindow();
}

void Processor::setCustomWindowCurve(const float* curve, size_t length) {
    if (!curve || length == 0) throw std::invalid_argument("Invalid custom window curve");
    impl->config.setCustomWindowCurve(curve, length);
    impl->config.windowingParams.useCustomCurve = true;
    impl->pushWindow();
}

void Processor::useCustomWindowCurve(bool useCustom) {
    if (useCustom && !impl->config.hasCustomWindowCurve())
        throw std::runtime_error("No custom window curve set. Call setCustomWindowCurve() first.");
    impl->config.windowingParams.useCustomCurve = useCustom;
    impl->pushWindow();
}

void Processor::enableWindowing(bool enable) {
    impl->config.windowingParams.enabled = enable;
    impl->pushConfig();
}

// ---- post-processing ------------------------------------------------------

void Processor::setGrayscaleRange(float min, float max) {
    impl->config.postProcessingParams.grayscaleMin = min;
    impl->config.postProcessingParams.grayscaleMax = max;
    impl->pushConfig();
}

void Processor::setSignalMultiplicatorAndAddend(float multiplicator, float addend) {
    impl->config.postProcessingParams.multiplicator = multiplicator;
    impl->config.postProcessingParams.addend = addend;
    impl->pushConfig();
}

void Processor::enableLogScaling(bool enable) {
    impl->config.postProcessingParams.logScaling = enable;
    impl->pushConfig();
}

void Processor::enableBackgroundRemoval(bool enable) {
    impl->config.backgroundRemovalParams.enabled = enable;
    impl->pushConfig();
}

void Processor::setBackgroundRemovalWindowSize(int windowSize) {
    impl->config.backgroundRemovalParams.rollingAverageWindowSize = windowSize;
    impl->pushConfig();
}

void Processor::enableBscanFlip(bool enable) {
    impl->config.postProcessingParams.bscanFlip = enable;
    impl->pushConfig();
}

void Processor::enableSinusoidalScanCorrection(bool enable) {
    impl->config.postProcessingParams.sinusoidalScanCorrection = enable;
    impl->pushConfig();
}

// ---- post-process background profile --------------------------------------

void Processor::requestPostProcessBackgroundRecording() {
    impl->ensureInitialized();
    impl->backend->requestPostProcessBackgroundRecording();
}

void Processor::setPostProcessBackgroundWeight(float weight) {
    impl->config.postProcessingParams.backgroundWeight = weight;
    impl->pushConfig();
}

void Processor::setPostProcessBackgroundOffset(float offset) {
    impl->config.postProcessingParams.backgroundOffset = offset;
    impl->pushConfig();
}

const float* Processor::getPostProcessBackgroundProfile() const {
    if (!impl->initialized) return impl->config.getCustomPostProcessBackgroundProfile();
    const auto& v = impl->backend->getPostProcessBackgroundProfile();
    return v.empty() ? nullptr : v.data();
}

size_t Processor::getPostProcessBackgroundProfileSize() const {
    if (!impl->initialized) return impl->config.getCustomPostProcessBackgroundProfileSize();
    return impl->backend->getPostProcessBackgroundProfile().size();
}

bool Processor::hasPostProcessBackgroundProfile() const {
    if (!impl->initialized) return impl->config.hasCustomPostProcessBackgroundProfile();
    return !impl->backend->getPostProcessBackgroundProfile().empty();
}

void Processor::setPostProcessBackgroundProfile(const float* data, size_t size) {
    if (!data || size == 0) throw std::invalid_argument("Invalid post-process background curve data");
    impl->config.setCustomPostProcessBackgroundProfile(data, size);
    if (impl->initialized) impl->backend->setPostProcessBackgroundProfile(data, size);
}

namespace {

// "<index>;<value>[;<value>]" lines after one header line (the reference's
// profile files, src/core/processor.cpp:640-700 and :782-832)
std::vector<float> read_profile_csv(const std::string& path, int values_per_line) {
    std::ifstream f(path);
    if (!f.is_open()) throw std::runtime_error("Failed to open file for reading: " + path);
    std::string line;
    if (!std::getline(f, line)) throw std::runtime_error("Empty file: " + path);
    std::vector<float> out;
    int lineno = 1;
    while (std::getline(f, line)) {
        ++lineno;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) continue;
        size_t pos = line.find(';');
        if (pos == std::string::npos)
            throw std::runtime_error("Invalid format at line " + std::to_string(lineno) + ": missing semicolon");
        for (int k = 0; k < values_per_line; ++k) {
            size_t next = (k + 1 < values_per_line) ? line.find(';', pos + 1) : std::string::npos;
            if (k + 1 < values_per_line && next == std::string::npos)
                throw std::runtime_error("Invalid format at line " + std::to_string(lineno));
            std::string tok = line.substr(pos + 1, next == std::string::npos ? std::string::npos : next - pos - 1);
            try {
                out.push_back(std::stof(tok));
            } catch (...) {
                throw std::runtime_error("Invalid number at line " + std::to_string(lineno) + ": " + tok);
            }
            pos = next;
        }
    }
    if (out.empty()) throw std::runtime_error("No data found in file: " + path);
    return out;
}

}  // namespace

void Processor::savePostProcessBackgroundProfileToFile(const std::string& filepath) const {
    const float* v = getPostProcessBackgroundProfile();
    const size_t n = getPostProcessBackgroundProfileSize();
    if (!v || n == 0) throw std::runtime_error("No post-process background curve to save");
    std::ofstream f(filepath);
    if (!f.is_open()) throw std::runtime_error("Failed to open file for writing: " + filepath);
    f << "Sample Number;Sample Value\n";
    for (size_t i = 0; i < n; ++i) f << i << ";" << v[i] << "\n";
    f.close();
    if (!f.good()) throw std::runtime_error("Error writing to file: " + filepath);
}

void Processor::loadPostProcessBackgroundProfileFromFile(const std::string& filepath) {
    auto v = read_profile_csv(filepath, 1);
    setPostProcessBackgroundProfile(v.data(), v.size());
}

void Processor::enablePostProcessBackgroundSubtraction(bool enable) {
    impl->config.postProcessingParams.backgroundRemoval = enable;
    impl->pushConfig();
}

// ---- fixed-pattern noise --------------------------------------------------

void Processor::enableFixedPatternNoiseRemoval(bool enable) {
    impl->config.postProcessingParams.fixedPatternNoiseRemoval = enable;
    impl->pushConfig();
}

void Processor::requestFixedPatternNoiseDetermination() {
    impl->ensureInitialized();
    impl->backend->requestFixedPatternNoiseDetermination();
}

void Processor::setFixedPatternNoiseBscanCount(int numberOfBscans) {
    if (numberOfBscans < 1) throw std::invalid_argument("numberOfBscans must be >= 1");
    impl->config.postProcessingParams.fixedPatternNoiseBscanCount = numberOfBscans;
    impl->pushConfig();
}

void Processor::enableContinuousFixedPatternNoiseDetermination(bool enable) {
    impl->config.postProcessingParams.continuousFixedPatternNoiseDetermination = enable;
    impl->pushConfig();
}

void Processor::setFixedPatternNoiseProfile(const float* data, size_t complexPairs) {
    if (!data || complexPairs == 0) throw std::invalid_argument("Invalid fixed pattern noise profile");
    impl->config.setCustomFixedPatternNoiseProfile(data, complexPairs);
    if (impl->initialized) impl->backend->setFixedPatternNoiseProfile(data, complexPairs);
}

const float* Processor::getFixedPatternNoiseProfile() const {
    if (!impl->initialized) return nullptr;
    const auto& v = impl->backend->getFixedPatternNoiseProfile();
    return v.empty() ? nullptr : v.data();
}

size_t Processor::getFixedPatternNoiseProfileSize() const {
    if (!impl->initialized) return 0;
    return impl->backend->getFixedPatternNoiseProfile().size() / 2;
}

bool Processor::hasFixedPatternNoiseProfile() const {
    if (!impl->initialized) return false;
    return !impl->backend->getFixedPatternNoiseProfile().empty();
}

void Processor::saveFixedPatternNoiseProfileToFile(const std::string& filepath) const {
    std::vector<float> v;
    if (impl->initialized) {
        v = impl->backend->getFixedPatternNoiseProfile();
    } else if (impl->config.hasCustomFixedPatternNoiseProfile()) {
        const float* p = impl->config.getCustomFixedPatternNoiseProfile();
        v.assign(p, p + 2 * impl->config.getCustomFixedPatternNoiseProfileSize());
    }
    if (v.empty()) throw std::runtime_error("No fixed pattern noise profile to save");
    std::ofstream f(filepath);
    if (!f.is_open()) throw std::runtime_error("Failed to open file for writing: " + filepath);
    f << "Sample Number;Real;Imag\n";
    for (size_t i = 0; i < v.size() / 2; ++i) f << i << ";" << v[2 * i] << ";" << v[2 * i + 1] << "\n";
    f.close();
    if (!f.good()) throw std::runtime_error("Error writing to file: " + filepath);
}

void Processor::loadFixedPatternNoiseProfileFromFile(const std::string& filepath) {
    auto v = read_profile_csv(filepath, 2);
    if (!impl->initialized)
        throw std::runtime_error("Processor must be initialized before loading fixed pattern noise profile");
    impl->backend->setFixedPatternNoiseProfile(v.data(), v.size() / 2);
}

// ---- low-level per-operation API -----------------------------------------

std::vector<float> Processor::convertInput(const void* input, IOBuffer::DataType inputType, int bitDepth, int samples,
                                           bool applyBitshift) {
    impl->ensureInitialized();
    return impl->backend->convertInput(input, inputType, bitDepth, samples, applyBitshift);
}
std::vector<float> Processor::rollingAverageBackgroundRemoval(const float* input, int windowSize, int lineWidth,
                                                              int numLines) {
    impl->ensureInitialized();
    return impl->backend->rollingAverageBackgroundRemoval(input, windowSize, lineWidth, numLines);
}
std::vector<float> Processor::kLinearization(const float* input, const float* resampleCurve,
                                             InterpolationMethod method, int lineWidth, int samples) {
    impl->ensureInitialized();
    return impl->backend->kLinearization(input, resampleCurve, method, lineWidth, samples);
}
std::vector<float> Processor::windowing(const float* input, const float* windowCurve, int lineWidth, int samples) {
    impl->ensureInitialized();
    return impl->backend->windowing(input, windowCurve, lineWidth, samples);
}
std::vector<float> Processor::dispersionCompensation(const float* input, const float* phaseComplex, int lineWidth,
                                                     int samples) {
    impl->ensureInitialized();
    return impl->backend->dispersionCompensation(input, phaseComplex, lineWidth, samples);
}
std::vector<float> Processor::kLinearizationAndWindowing(const float* input, const float* resampleCurve,
                                                         const float* windowCurve, InterpolationMethod method,
                                                         int lineWidth, int samples) {
    impl->ensureInitialized();
    return impl->backend->kLinearizationAndWindowing(input, resampleCurve, windowCurve, method, lineWidth, samples);
}
std::vector<float> Processor::kLinearizationAndWindowingAndDispersion(const float* input, const float* resampleCurve,
                                                                      const float* windowCurve,
                                                                      const float* phaseComplex,
                                                                      InterpolationMethod method, int lineWidth,
                                                                      int samples) {
    impl->ensureInitialized();
    return impl->backend->kLinearizationAndWindowingAndDispersion(input, resampleCurve, windowCurve, phaseComplex,
                                                                  method, lineWidth, samples);
}
std::vector<float> Processor::dispersionCompensationAndWindowing(const float* input, const float* phaseComplex,
                                                                 const float* windowCurve, int lineWidth,
                                                                 int samples) {
    impl->ensureInitialized();
    return impl->backend->dispersionCompensationAndWindowing(input, phaseComplex, windowCurve, lineWidth, samples);
}
std::vector<float> Processor::fft(const float* input, int lineWidth, int samples) {
    impl->ensureInitialized();
    return impl->backend->fft(input, lineWidth, samples);
}
std::vector<float> Processor::ifft(const float* input, int lineWidth, int samples) {
    impl->ensureInitialized();
    return impl->backend->ifft(input, lineWidth, samples);
}
std::vector<float> Processor::getMinimumVarianceMean(const float* input, int width, int height, int segments) {
    impl->ensureInitialized();
    return impl->backend->getMinimumVarianceMean(input, width, height, segments);
}
std::vector<float> Processor::fixedPatternNoiseRemoval(const float* input, const float* meanALine, int lineWidth,
                                                       int numLines) {
    impl->ensureInitialized();
    return impl->backend->fixedPatternNoiseRemoval(input, meanALine, lineWidth, numLines);
}
std::vector<float> Processor::postProcessTruncate(const float* input, bool logScaling, float grayscaleMax,
                                                  float grayscaleMin, float addend, float multiplicator,
                                                  int lineWidth, int samples) {
    impl->ensureInitialized();
    return impl->backend->postProcessTruncate(input, logScaling, grayscaleMax, grayscaleMin, addend, multiplicator,
                                              lineWidth, samples);
}
std::vector<float> Processor::bscanFlip(const float* input, int lineWidth, int linesPerBscan, int numBscans) {
    impl->ensureInitialized();
    return impl->backend->bscanFlip(input, lineWidth, linesPerBscan, numBscans);
}
std::vector<float> Processor::sinusoidalScanCorrection(const float* input, const float* resampleCurve,
                                                       int lineWidth, int linesPerBscan, int numBscans) {
    impl->ensureInitialized();
    return impl->backend->sinusoidalScanCorrection(input, resampleCurve, lineWidth, linesPerBscan, numBscans);
}
std::vector<float> Processor::postProcessBackgroundSubtraction(const float* input, const float* backgroundLine,
                                                               float weight, float offset, int lineWidth,
                                                               int samples) {
    impl->ensureInitialized();
    return impl->backend->postProcessBackgroundSubtraction(input, backgroundLine, weight, offset, lineWidth,
                                                           samples);
}

}  // namespace ope
