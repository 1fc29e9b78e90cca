// ProcessorConfiguration: custom curves (kept as given and as adjusted to the
// signal length), generated curves (the library's bit-identical generators,
// include/ope_b200.h) and INI-style persistence.
#include "../../include/ope/processorconfiguration.h"

#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <vector>

#include "../../include/ope_b200.h"

namespace ope {

struct ProcessorConfiguration::Impl {
    // [0] resampling, [1] window, [2] dispersion phase, [3] post-process background, [4] FPN (interleaved)
    std::vector<float> original[5];
    std::vector<float> adjusted[5];
    mutable std::vector<float> generated[3];
};

namespace {
enum { RES = 0, WIN = 1, DISP = 2, BG = 3, FPN = 4 };

void set_curve(std::vector<float>& orig, const float* data, size_t n, const char* what) {
    if (!data) throw std::invalid_argument(std::string("Custom ") + what + " data is null");
    if (n == 0) throw std::invalid_argument(std::string("Custom ") + what + " size is zero");
    orig.assign(data, data + n);
}
}  // namespace

ProcessorConfiguration::ProcessorConfiguration() : impl(new Impl()) {}
ProcessorConfiguration::~ProcessorConfiguration() { delete impl; }
ProcessorConfiguration::ProcessorConfiguration(const ProcessorConfiguration& o)
    : dataParams(o.dataParams), processingParams(o.processingParams), resamplingParams(o.resamplingParams),
      windowingParams(o.windowingParams), dispersionParams(o.dispersionParams),
      backgroundRemovalParams(o.backgroundRemovalParams), postProcessingParams(o.postProcessingParams),
      impl(new Impl(*o.impl)) {}
ProcessorConfiguration::ProcessorConfiguration(ProcessorConfiguration&& o) noexcept
    : dataParams(o.dataParams), processingParams(o.processingParams), resamplingParams(o.resamplingParams),
      windowingParams(o.windowingParams), dispersionParams(o.dispersionParams),
      backgroundRemovalParams(o.backgroundRemovalParams), postProcessingParams(o.postProcessingParams),
      impl(o.impl) {
    o.impl = new Impl();
}
ProcessorConfiguration& ProcessorConfiguration::operator=(const ProcessorConfiguration& o) {
    if (this != &o) {
        dataParams = o.dataParams;
        processingParams = o.processingParams;
        resamplingParams = o.resamplingParams;
        windowingParams = o.windowingParams;
        dispersionParams = o.dispersionParams;
        backgroundRemovalParams = o.backgroundRemovalParams;
        postProcessingParams = o.postProcessingParams;
        *impl = *o.impl;
    }
    return *this;
}
ProcessorConfiguration& ProcessorConfiguration::operator=(ProcessorConfiguration&& o) noexcept {
    if (this != &o) {
        dataParams = o.dataParams;
        processingParams = o.processingParams;
        resamplingParams = o.resamplingParams;
        windowingParams = o.windowingParams;
        dispersionParams = o.dispersionParams;
        backgroundRemovalParams = o.backgroundRemovalParams;
        postProcessingParams = o.postProcessingParams;
        std::swap(impl, o.impl);
    }
    return *this;
}

void ProcessorConfiguration::setCustomResamplingCurve(const float* d, size_t n) {
    set_curve(impl->original[RES], d, n, "resampling curve");
    adjustAllCustomCurves();
}
void ProcessorConfiguration::setCustomWindowCurve(const float* d, size_t n) {
    set_curve(impl->original[WIN], d, n, "window curve");
    adjustAllCustomCurves();
}
void ProcessorConfiguration::setCustomDispersionCurve(const float* d, size_t n) {
    set_curve(impl->original[DISP], d, n, "dispersion curve");
    adjustAllCustomCurves();
}
void ProcessorConfiguration::setCustomPostProcessBackgroundProfile(const float* d, size_t n) {
    set_curve(impl->original[BG], d, n, "post-process background curve");
    adjustAllCustomCurves();
}
void ProcessorConfiguration::setCustomFixedPatternNoiseProfile(const float* d, size_t pairs) {
    set_curve(impl->original[FPN], d, pairs * 2, "fixed-pattern noise profile");
    adjustAllCustomCurves();
}

static const float* data_or_null(const std::vector<float>& v) { return v.empty() ? nullptr : v.data(); }
const float* ProcessorConfiguration::getCustomResamplingCurve() const { return data_or_null(impl->adjusted[RES]); }
const float* ProcessorConfiguration::getCustomWindowCurve() const { return data_or_null(impl->adjusted[WIN]); }
const float* ProcessorConfiguration::getCustomDispersionCurve() const { return data_or_null(impl->adjusted[DISP]); }
const float* ProcessorConfiguration::getCustomPostProcessBackgroundProfile() const {
    return data_or_null(impl->adjusted[BG]);
}
const float* ProcessorConfiguration::getCustomFixedPatternNoiseProfile() const {
    return data_or_null(impl->adjusted[FPN]);
}
size_t ProcessorConfiguration::getCustomResamplingCurveSize() const { return impl->adjusted[RES].size(); }
size_t ProcessorConfiguration::getCustomWindowCurveSize() const { return impl->adjusted[WIN].size(); }
size_t ProcessorConfiguration::getCustomDispersionCurveSize() const { return impl->adjusted[DISP].size(); }
size_t ProcessorConfiguration::getCustomPostProcessBackgroundProfileSize() const { return impl->adjusted[BG].size(); }
size_t ProcessorConfiguration::getCustomFixedPatternNoiseProfileSize() const { return impl->adjusted[FPN].size() / 2; }
bool ProcessorConfiguration::hasCustomResamplingCurve() const { return !impl->original[RES].empty(); }
bool ProcessorConfiguration::hasCustomWindowCurve() const { return !impl->original[WIN].empty(); }
bool ProcessorConfiguration::hasCustomDispersionCurve() const { return !impl->original[DISP].empty(); }
bool ProcessorConfiguration::hasCustomPostProcessBackgroundProfile() const { return !impl->original[BG].empty(); }
bool ProcessorConfiguration::hasCustomFixedPatternNoiseProfile() const { return !impl->original[FPN].empty(); }

const float* ProcessorConfiguration::getGeneratedResamplingCurve() const {
    auto& g = impl->generated[RES];
    g.resize(static_cast<size_t>(dataParams.signalLength));
    ope_b200_generate_resampling_curve(dataParams.signalLength, resamplingParams.coefficients, g.data());
    return g.data();
}
const float* ProcessorConfiguration::getGeneratedWindowCurve() const {
    auto& g = impl->generated[WIN];
    g.resize(static_cast<size_t>(dataParams.signalLength));
    ope_b200_generate_window_curve(dataParams.signalLength, static_cast<int>(windowingParams.windowType),
                                   windowingParams.windowCenterPosition, windowingParams.windowFillFactor, g.data());
    return g.data();
}
const float* ProcessorConfiguration::getGeneratedDispersionCurve() const {
    auto& g = impl->generated[DISP];
    g.resize(static_cast<size_t>(dataParams.signalLength));
    ope_b200_generate_dispersion_phase(dataParams.signalLength, dispersionParams.coefficients, g.data());
    return g.data();
}
size_t ProcessorConfiguration::getGeneratedResamplingCurveSize() const { return dataParams.signalLength; }
size_t ProcessorConfiguration::getGeneratedWindowCurveSize() const { return dataParams.signalLength; }
size_t ProcessorConfiguration::getGeneratedDispersionCurveSize() const { return dataParams.signalLength; }

// Custom curves are zero-padded or truncated to the signal length (N values;
// N/2 for the background profile, N/2 complex pairs for the FPN profile), as
// the reference does (processorconfiguration.cpp:268-432).
void ProcessorConfiguration::adjustAllCustomCurves() {
    const size_t n = static_cast<size_t>(dataParams.signalLength > 0 ? dataParams.signalLength : 0);
    const size_t target[5] = {n, n, n, n / 2, (n / 2) * 2};
    for (int k = 0; k < 5; ++k) {
        impl->adjusted[k] = impl->original[k];
        if (!impl->adjusted[k].empty()) impl->adjusted[k].resize(target[k], 0.0f);
    }
}

bool ProcessorConfiguration::validate() const {
    return dataParams.signalLength > 0 && dataParams.samplesPerBuffer > 0 && dataParams.ascansPerBscan > 0 &&
           dataParams.bscansPerBuffer > 0;
}

// ---- INI persistence: [section] key=value, curves as comma-separated floats ----

namespace {
std::string join(const std::vector<float>& v) {
    std::ostringstream os;
    os.precision(9);
    for (size_t i = 0; i < v.size(); ++i) os << (i ? "," : "") << v[i];
    return os.str();
}
std::vector<float> split(const std::string& s) {
    std::vector<float> v;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, ','))
        if (!tok.empty()) v.push_back(std::stof(tok));
    return v;
}
}  // namespace

bool ProcessorConfiguration::saveToFile(const std::string& filepath) const {
    std::ofstream f(filepath);
    if (!f.is_open()) return false;
    f.precision(9);
    const auto& d = dataParams;
    f << "[data]\nsignalLength=" << d.signalLength << "\nascansPerBscan=" << d.ascansPerBscan
      << "\nbscansPerBuffer=" << d.bscansPerBuffer << "\nsamplesPerBuffer=" << d.samplesPerBuffer
      << "\ninputDataType=" << static_cast<int>(d.inputDataType) << "\nbitshift=" << d.bitshift << "\n";
    const auto& p = processingParams;
    f << "[processing]\nnStreams=" << p.nStreams << "\nnBuffers=" << p.nBuffers << "\ngridSize=" << p.gridSize
      << "\nblockSize=" << p.blockSize << "\n";
    const auto& r = resamplingParams;
    f << "[resampling]\nenabled=" << r.enabled << "\ninterpolationMethod=" << static_cast<int>(r.interpolationMethod)
      << "\nuseCoefficients=" << r.useCoefficients << "\ncoefficients="
      << join(std::vector<float>(r.coefficients, r.coefficients + 4)) << "\nuseCustomCurve=" << r.useCustomCurve
      << "\ncustomCurve=" << join(impl->original[RES]) << "\n";
    const auto& w = windowingParams;
    f << "[windowing]\nenabled=" << w.enabled << "\nwindowType=" << static_cast<int>(w.windowType)
      << "\nwindowCenterPosition=" << w.windowCenterPosition << "\nwindowFillFactor=" << w.windowFillFactor
      << "\nuseCustomCurve=" << w.useCustomCurve << "\ncustomCurve=" << join(impl->original[WIN]) << "\n";
    const auto& q = dispersionParams;
    f << "[dispersion]\nenabled=" << q.enabled << "\nuseCoefficients=" << q.useCoefficients << "\ncoefficients="
      << join(std::vector<float>(q.coefficients, q.coefficients + 4)) << "\nfactor=" << q.factor
      << "\nuseCustomCurve=" << q.useCustomCurve << "\ncustomCurve=" << join(impl->original[DISP]) << "\n";
    const auto& b = backgroundRemovalParams;
    f << "[backgroundRemoval]\nenabled=" << b.enabled << "\nrollingAverageWindowSize=" << b.rollingAverageWindowSize
      << "\n";
    const auto& o = postProcessingParams;
    f << "[postProcessing]\nbackgroundRemoval=" << o.backgroundRemoval << "\nbackgroundWeight=" << o.backgroundWeight
      << "\nbackgroundOffset=" << o.backgroundOffset << "\nlogScaling=" << o.logScaling << "\ngrayscaleMax="
      << o.grayscaleMax << "\ngrayscaleMin=" << o.grayscaleMin << "\naddend=" << o.addend << "\nmultiplicator="
      << o.multiplicator << "\nbscanFlip=" << o.bscanFlip << "\nsinusoidalScanCorrection="
      << o.sinusoidalScanCorrection << "\nfixedPatternNoiseRemoval=" << o.fixedPatternNoiseRemoval
      << "\nfixedPatternNoiseBscanCount=" << o.fixedPatternNoiseBscanCount
      << "\ncontinuousFixedPatternNoiseDetermination=" << o.continuousFixedPatternNoiseDetermination
      << "\nbackgroundProfile=" << join(impl->original[BG]) << "\nfixedPatternNoiseProfile="
      << join(impl->original[FPN]) << "\n";
    return f.good();
}

bool ProcessorConfiguration::loadFromFile(const std::string& filepath) {
    std::ifstream f(filepath);
    if (!f.is_open()) return false;
    std::map<std::string, std::string> kv;
    std::string line, section;
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty() || line[0] == ';' || line[0] == '#') continue;
        if (line.front() == '[' && line.back() == ']') {
            section = line.substr(1, line.size() - 2);
            continue;
        }
        const size_t eq = line.find('=');
        if (eq == std::string::npos) return false;
        kv[section + "." + line.substr(0, eq)] = line.substr(eq + 1);
    }
    try {
        ProcessorConfiguration c;
        auto geti = [&](const char* k, int& dst) {
            auto it = kv.find(k);
            if (it != kv.end()) dst = std::stoi(it->second);
        };
        auto getb = [&](const char* k, bool& dst) {
            auto it = kv.find(k);
            if (it != kv.end()) dst = std::stoi(it->second) != 0;
        };
        auto getf = [&](const char* k, float& dst) {
            auto it = kv.find(k);
            if (it != kv.end()) dst = std::stof(it->second);
        };
        auto getv = [&](const char* k) {
            auto it = kv.find(k);
            return it == kv.end() ? std::vector<float>() : split(it->second);
        };
        int t = 0;
        geti("data.signalLength", c.dataParams.signalLength);
        geti("data.ascansPerBscan", c.dataParams.ascansPerBscan);
        geti("data.bscansPerBuffer", c.dataParams.bscansPerBuffer);
        geti("data.samplesPerBuffer", c.dataParams.samplesPerBuffer);
        t = static_cast<int>(c.dataParams.inputDataType);
        geti("data.inputDataType", t);
        c.dataParams.inputDataType = static_cast<DataType>(t);
        getb("data.bitshift", c.dataParams.bitshift);
        geti("processing.nStreams", c.processingParams.nStreams);
        geti("processing.nBuffers", c.processingParams.nBuffers);
        geti("processing.gridSize", c.processingParams.gridSize);
        geti("processing.blockSize", c.processingParams.blockSize);
        getb("resampling.enabled", c.resamplingParams.enabled);
        t = static_cast<int>(c.resamplingParams.interpolationMethod);
        geti("resampling.interpolationMethod", t);
        c.resamplingParams.interpolationMethod = static_cast<InterpolationMethod>(t);
        getb("resampling.useCoefficients", c.resamplingParams.useCoefficients);
        getb("resampling.useCustomCurve", c.resamplingParams.useCustomCurve);
        auto rc = getv("resampling.coefficients");
        for (size_t i = 0; i < 4 && i < rc.size(); ++i) c.resamplingParams.coefficients[i] = rc[i];
        getb("windowing.enabled", c.windowingParams.enabled);
        t = static_cast<int>(c.windowingParams.windowType);
        geti("windowing.windowType", t);
        c.windowingParams.windowType = static_cast<WindowType>(t);
        getf("windowing.windowCenterPosition", c.windowingParams.windowCenterPosition);
        getf("windowing.windowFillFactor", c.windowingParams.windowFillFactor);
        getb("windowing.useCustomCurve", c.windowingParams.useCustomCurve);
        getb("dispersion.enabled", c.dispersionParams.enabled);
        getb("dispersion.useCoefficients", c.dispersionParams.useCoefficients);
        auto dc = getv("dispersion.coefficients");
        for (size_t i = 0; i < 4 && i < dc.size(); ++i) c.dispersionParams.coefficients[i] = dc[i];
        getf("dispersion.factor", c.dispersionParams.factor);
        getb("dispersion.useCustomCurve", c.dispersionParams.useCustomCurve);
        getb("backgroundRemoval.enabled", c.backgroundRemovalParams.enabled);
        geti("backgroundRemoval.rollingAverageWindowSize", c.backgroundRemovalParams.rollingAverageWindowSize);
        auto& pp = c.postProcessingParams;
        getb("postProcessing.backgroundRemoval", pp.backgroundRemoval);
        getf("postProcessing.backgroundWeight", pp.backgroundWeight);
        getf("postProcessing.backgroundOffset", pp.backgroundOffset);
        getb("postProcessing.logScaling", pp.logScaling);
        getf("postProcessing.grayscaleMax", pp.grayscaleMax);
        getf("postProcessing.grayscaleMin", pp.grayscaleMin);
        getf("postProcessing.addend", pp.addend);
        getf("postProcessing.multiplicator", pp.multiplicator);
        getb("postProcessing.bscanFlip", pp.bscanFlip);
        getb("postProcessing.sinusoidalScanCorrection", pp.sinusoidalScanCorrection);
        getb("postProcessing.fixedPatternNoiseRemoval", pp.fixedPatternNoiseRemoval);
        geti("postProcessing.fixedPatternNoiseBscanCount", pp.fixedPatternNoiseBscanCount);
        getb("postProcessing.continuousFixedPatternNoiseDetermination", pp.continuousFixedPatternNoiseDetermination);
        c.impl->original[RES] = getv("resampling.customCurve");
        c.impl->original[WIN] = getv("windowing.customCurve");
        c.impl->original[DISP] = getv("dispersion.customCurve");
        c.impl->original[BG] = getv("postProcessing.backgroundProfile");
        c.impl->original[FPN] = getv("postProcessing.fixedPatternNoiseProfile");
        c.adjustAllCustomCurves();
        *this = c;
    } catch (const std::exception&) {
        return false;
    }
    return true;
}

}  // namespace ope
