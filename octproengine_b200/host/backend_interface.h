// The backend seam of the OCTproEngine Processor: the methods a processing
// backend provides (the same set as the reference's ProcessingBackend,
// src/backends/backend_interface.h:12-165), declared here for this build.
#pragma once

#include <functional>
#include <vector>

#include "../../include/ope/iobuffer.h"
#include "../../include/ope/processorconfiguration.h"

namespace ope {

class ProcessingBackend {
public:
    virtual ~ProcessingBackend() = default;

    virtual void initialize(const ProcessorConfiguration& config) = 0;
    virtual void cleanup() = 0;
    virtual void setOutputCallback(std::function<void(const IOBuffer&)> callback) = 0;
    virtual void process(IOBuffer& input) = 0;
    virtual void updateConfig(const ProcessorConfiguration& config) = 0;
    virtual void updateResamplingCurve(const float* curve, size_t length) = 0;
    virtual void updateDispersionCurve(const float* curve, size_t length) = 0;
    virtual void updateWindowCurve(const float* curve, size_t length) = 0;
    virtual IOBuffer& getInputBuffer(int index) = 0;
    virtual IOBuffer& getNextAvailableInputBuffer() = 0;
    virtual int getNumInputBuffers() const = 0;
    virtual void requestPostProcessBackgroundRecording() = 0;
    virtual void setPostProcessBackgroundProfile(const float* background, size_t length) = 0;
    virtual const std::vector<float>& getPostProcessBackgroundProfile() const = 0;
    virtual void requestFixedPatternNoiseDetermination() = 0;
    virtual void setFixedPatternNoiseProfile(const float* profileInterleaved, size_t complexPairs) = 0;
    virtual const std::vector<float>& getFixedPatternNoiseProfile() const = 0;

    virtual std::vector<float> convertInput(const void* input, IOBuffer::DataType inputType, int bitDepth,
                                            int samples, bool applyBitshift) = 0;
    virtual std::vector<float> rollingAverageBackgroundRemoval(const float* input, int windowSize, int lineWidth,
                                                               int numLines) = 0;
    virtual std::vector<float> kLinearization(const float* input, const float* resampleCurve,
                                              InterpolationMethod method, int lineWidth, int samples) = 0;
    virtual std::vector<float> windowing(const float* input, const float* windowCurve, int lineWidth,
                                         int samples) = 0;
    virtual std::vector<float> dispersionCompensation(const float* input, const float* phaseComplex, int lineWidth,
                                                      int samples) = 0;
    virtual std::vector<float> kLinearizationAndWindowing(const float* input, const float* resampleCurve,
                                                          const float* windowCurve, InterpolationMethod method,
                                                          int lineWidth, int samples) = 0;
    virtual std::vector<float> kLinearizationAndWindowingAndDispersion(const float* input, const float* resampleCurve,
                                                                       const float* windowCurve,
                                                                       const float* phaseComplex,
                                                                       InterpolationMethod method, int lineWidth,
                                                                       int samples) = 0;
    virtual std::vector<float> dispersionCompensationAndWindowing(const float* input, const float* phaseComplex,
                                                                  const float* windowCurve, int lineWidth,
                                                                  int samples) = 0;
    virtual std::vector<float> fft(const float* input, int lineWidth, int samples) = 0;
    virtual std::vector<float> ifft(const float* input, int lineWidth, int samples) = 0;
    virtual std::vector<float> getMinimumVarianceMean(const float* input, int width, int height, int segments) = 0;
    virtual std::vector<float> fixedPatternNoiseRemoval(const float* input, const float* meanALine, int lineWidth,
                                                        int numLines) = 0;
    virtual std::vector<float> postProcessTruncate(const float* input, bool logScaling, float grayscaleMax,
                                                   float grayscaleMin, float addend, float multiplicator,
                                                   int lineWidth, int samples) = 0;
    virtual std::vector<float> bscanFlip(const float* input, int lineWidth, int linesPerBscan, int numBscans) = 0;
    virtual std::vector<float> sinusoidalScanCorrection(const float* input, const float* resampleCurve,
                                                        int lineWidth, int linesPerBscan, int numBscans) = 0;
    virtual std::vector<float> postProcessBackgroundSubtraction(const float* input, const float* backgroundLine,
                                                                float weight, float offset, int lineWidth,
                                                                int samples) = 0;
};

}  // namespace ope
