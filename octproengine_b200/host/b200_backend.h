// ope::B200Backend: the ProcessingBackend of this build. Every method forwards
// to the C ABI of include/ope_b200.h; a non-zero status becomes
// std::runtime_error (std::invalid_argument for argument errors), the
// reference backends' convention.
#pragma once

#include <memory>

// Built into the reference library (the Backend::B200 patch), the class derives
// from the reference's own ProcessingBackend: that build names its
// src/backends/backend_interface.h here. This library's own host layer uses the
// interface declared beside this file.
#if defined(OPE_B200_REFERENCE_INTERFACE)
#include OPE_B200_REFERENCE_INTERFACE
#else
#include "backend_interface.h"
#endif

namespace ope {

class B200Backend : public ProcessingBackend {
public:
    B200Backend();
    ~B200Backend() override;

    void initialize(const ProcessorConfiguration& config) override;
    void cleanup() override;
    void setOutputCallback(std::function<void(const IOBuffer&)> callback) override;
    void process(IOBuffer& input) override;
    void updateConfig(const ProcessorConfiguration& config) override;
    void updateResamplingCurve(const float* curve, size_t length) override;
    void updateDispersionCurve(const float* curve, size_t length) override;
    void updateWindowCurve(const float* curve, size_t length) override;
    IOBuffer& getInputBuffer(int index) override;
    IOBuffer& getNextAvailableInputBuffer() override;
    int getNumInputBuffers() const override;
    void requestPostProcessBackgroundRecording() override;
    void setPostProcessBackgroundProfile(const float* background, size_t length) override;
    const std::vector<float>& getPostProcessBackgroundProfile() const override;
    void requestFixedPatternNoiseDetermination() override;
    void setFixedPatternNoiseProfile(const float* profileInterleaved, size_t complexPairs) override;
    const std::vector<float>& getFixedPatternNoiseProfile() const override;

    std::vector<float> convertInput(const void* input, IOBuffer::DataType inputType, int bitDepth, int samples,
                                    bool applyBitshift) override;
    std::vector<float> rollingAverageBackgroundRemoval(const float* input, int windowSize, int lineWidth,
                                                       int numLines) override;
    std::vector<float> kLinearization(const float* input, const float* resampleCurve, InterpolationMethod method,
                                      int lineWidth, int samples) override;
    std::vector<float> windowing(const float* input, const float* windowCurve, int lineWidth, int samples) override;
    std::vector<float> dispersionCompensation(const float* input, const float* phaseComplex, int lineWidth,
                                              int samples) override;
    std::vector<float> kLinearizationAndWindowing(const float* input, const float* resampleCurve,
                                                  const float* windowCurve, InterpolationMethod method, int lineWidth,
                                                  int samples) override;
    std::vector<float> kLinearizationAndWindowingAndDispersion(const float* input, const float* resampleCurve,
                                                               const float* windowCurve, const float* phaseComplex,
                                                               InterpolationMethod method, int lineWidth,
                                                               int samples) override;
    std::vector<float> dispersionCompensationAndWindowing(const float* input, const float* phaseComplex,
                                                          const float* windowCurve, int lineWidth,
                                                          int samples) override;
    std::vector<float> fft(const float* input, int lineWidth, int samples) override;
    std::vector<float> ifft(const float* input, int lineWidth, int samples) override;
    std::vector<float> getMinimumVarianceMean(const float* input, int width, int height, int segments) override;
    std::vector<float> fixedPatternNoiseRemoval(const float* input, const float* meanALine, int lineWidth,
                                                int numLines) override;
    std::vector<float> postProcessTruncate(const float* input, bool logScaling, float grayscaleMax,
                                           float grayscaleMin, float addend, float multiplicator, int lineWidth,
                                           int samples) override;
    std::vector<float> bscanFlip(const float* input, int lineWidth, int linesPerBscan, int numBscans) override;
    std::vector<float> sinusoidalScanCorrection(const float* input, const float* resampleCurve, int lineWidth,
                                                int linesPerBscan, int numBscans) override;
    std::vector<float> postProcessBackgroundSubtraction(const float* input, const float* backgroundLine,
                                                        float weight, float offset, int lineWidth,
                                                        int samples) override;

    // Rolling-average DC removal. true (the default): the reference CPU
    // backend's sequential float prefix sum, so a frame with background
    // removal on equals that backend's output bit for bit up to the DFT;
    // false: exact integer window sums (the exact mean of each window).
    // Takes effect at the next initialize() or updateConfig().
    void setRollingAverageReferenceOrder(bool on);

private:
    struct Impl;
    std::unique_ptr<Impl> impl;
};

}  // namespace ope
