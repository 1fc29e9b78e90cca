// The processing facade of the OCTproEngine API (reference include/processor.h:14-287):
// the same methods with the same argument meaning, driving the B200 backend.
#ifndef OPE_B200_PROCESSOR_H
#define OPE_B200_PROCESSOR_H

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "export.h"
#include "iobuffer.h"
#include "processorconfiguration.h"

namespace ope {

class OPE_API Processor {
public:
    using OutputCallback = std::function<void(const IOBuffer&)>;
    using CallbackId = int;

    explicit Processor(Backend backend);
    ~Processor();
    Processor(const Processor&) = delete;
    Processor& operator=(const Processor&) = delete;

    void initialize();
    void cleanup();
    bool isInitialized() const;

    void loadConfigurationFromFile(const std::string& filepath);
    void saveConfigurationToFile(const std::string& filepath) const;

    const ProcessorConfiguration& getConfig() const;
    void setConfig(const ProcessorConfiguration& config);

    void setInputParameters(int samplesPerRawAscan, int ascansPerBscan, int bscansPerBuffer, DataType type);

    void setBackend(Backend backend);
    Backend getBackend() const;

    // asynchronous: the output arrives through the registered callbacks
    void process(IOBuffer& input);

    void setOutputCallback(OutputCallback callback);
    CallbackId addOutputCallback(OutputCallback callback);
    bool removeOutputCallback(CallbackId id);
    void clearOutputCallbacks();
    size_t getCallbackCount() const;

    IOBuffer& getInputBuffer(int index);
    int getNumInputBuffers() const;
    IOBuffer& getNextAvailableInputBuffer();

    // hot-swap: resampling
    void setResamplingCoefficients(const float coefficients[4]);
    void setCustomResamplingCurve(const float* curve, size_t length);
    void useCustomResamplingCurve(bool useCustom);
    void enableResampling(bool enable);
    void setInterpolationMethod(InterpolationMethod method);

    // hot-swap: dispersion
    void setDispersionCoefficients(const float coefficients[4], float factor = 1.0f);
    void setCustomDispersionCurve(const float* curve, size_t length);
    void useCustomDispersionCurve(bool useCustom);
    void enableDispersionCompensation(bool enable);

    // hot-swap: windowing
    void setWindowParameters(WindowType type, float centerPosition, float fillFactor);
    void setCustomWindowCurve(const float* curve, size_t length);
    void useCustomWindowCurve(bool useCustom);
    void enableWindowing(bool enable);

    // post-processing
    void setGrayscaleRange(float min, float max);
    void setSignalMultiplicatorAndAddend(float multiplicator, float addend);
    void enableLogScaling(bool enable);

    // rolling-average DC (background) removal
    void enableBackgroundRemoval(bool enable);
    void setBackgroundRemovalWindowSize(int windowSize);

    // post-process background profile subtraction
    void requestPostProcessBackgroundRecording();
    void setPostProcessBackgroundWeight(float weight);
    void setPostProcessBackgroundOffset(float offset);
    const float* getPostProcessBackgroundProfile() const;
    size_t getPostProcessBackgroundProfileSize() const;
    bool hasPostProcessBackgroundProfile() const;
    void setPostProcessBackgroundProfile(const float* data, size_t size);
    void savePostProcessBackgroundProfileToFile(const std::string& filepath) const;
    void loadPostProcessBackgroundProfileFromFile(const std::string& filepath);
    void enablePostProcessBackgroundSubtraction(bool enable);

    void enableBscanFlip(bool enable);
    void enableSinusoidalScanCorrection(bool enable);

    // fixed-pattern noise
    void enableFixedPatternNoiseRemoval(bool enable);
    void requestFixedPatternNoiseDetermination();
    void setFixedPatternNoiseBscanCount(int numberOfBscans);
    void enableContinuousFixedPatternNoiseDetermination(bool enable);
    void setFixedPatternNoiseProfile(const float* data, size_t complexPairs);
    const float* getFixedPatternNoiseProfile() const;
    size_t getFixedPatternNoiseProfileSize() const;
    bool hasFixedPatternNoiseProfile() const;
    void saveFixedPatternNoiseProfileToFile(const std::string& filepath) const;
    void loadFixedPatternNoiseProfileFromFile(const std::string& filepath);

    // low-level per-operation API (for testing)
    std::vector<float> convertInput(const void* input, IOBuffer::DataType inputType, int bitDepth, int samples,
                                    bool applyBitshift = false);
    std::vector<float> rollingAverageBackgroundRemoval(const float* input, int windowSize, int lineWidth,
                                                       int numLines);
    std::vector<float> kLinearization(const float* input, const float* resampleCurve, InterpolationMethod method,
                                      int lineWidth, int samples);
    std::vector<float> windowing(const float* input, const float* windowCurve, int lineWidth, int samples);
    std::vector<float> dispersionCompensation(const float* input, const float* phaseComplex, int lineWidth,
                                              int samples);
    std::vector<float> kLinearizationAndWindowing(const float* input, const float* resampleCurve,
                                                  const float* windowCurve, InterpolationMethod method, int lineWidth,
                                                  int samples);
    std::vector<float> kLinearizationAndWindowingAndDispersion(const float* input, const float* resampleCurve,
                                                               const float* windowCurve, const float* phaseComplex,
                                                               InterpolationMethod method, int lineWidth, int samples);
    std::vector<float> dispersionCompensationAndWindowing(const float* input, const float* phaseComplex,
                                                          const float* windowCurve, int lineWidth, int samples);
    std::vector<float> fft(const float* input, int lineWidth, int samples);
    std::vector<float> ifft(const float* input, int lineWidth, int samples);
    std::vector<float> getMinimumVarianceMean(const float* input, int width, int height, int segments);
    std::vector<float> fixedPatternNoiseRemoval(const float* input, const float* meanALine, int lineWidth,
                                                int numLines);
    std::vector<float> postProcessTruncate(const float* input, bool logScaling, float grayscaleMax,
                                           float grayscaleMin, float addend, float multiplicator, int lineWidth,
                                           int samples);
    std::vector<float> bscanFlip(const float* input, int lineWidth, int linesPerBscan, int numBscans);
    std::vector<float> sinusoidalScanCorrection(const float* input, const float* resampleCurve, int lineWidth,
                                                int linesPerBscan, int numBscans);
    std::vector<float> postProcessBackgroundSubtraction(const float* input, const float* backgroundLine,
                                                        float weight, float offset, int lineWidth, int samples);

private:
    class Impl;
    std::unique_ptr<Impl> impl;
};

}  // namespace ope

#endif
