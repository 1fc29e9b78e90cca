// Python module `octproengine` over the C++ host layer: the names, argument
// order, exceptions and buffer semantics of the reference's Python binding
// (python/octproengine_bindings.cpp), so scripts written for it run unchanged
// with Backend.CUDA (or Backend.B200) selecting the sm_100a backend.
//
// Buffers cross as zero-copy NumPy views of ope::IOBuffer memory: an input
// view from get_next_available_buffer() is handed back to process(); an output
// view passed to a callback is valid while the callback runs.
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "ope/iobuffer.h"
#include "ope/processor.h"
#include "ope/processorconfiguration.h"
#include "ope/types.h"

namespace py = pybind11;

namespace {

struct InitializationError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ConfigurationError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct BufferError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ProcessingError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct BackendError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

py::dtype numpy_dtype(ope::DataType t) {
    switch (t) {
        case ope::DataType::UINT8: return py::dtype::of<uint8_t>();
        case ope::DataType::UINT16: return py::dtype::of<uint16_t>();
        case ope::DataType::UINT32: return py::dtype::of<uint32_t>();
        case ope::DataType::INT8: return py::dtype::of<int8_t>();
        case ope::DataType::INT16: return py::dtype::of<int16_t>();
        case ope::DataType::INT32: return py::dtype::of<int32_t>();
        case ope::DataType::FLOAT32: return py::dtype::of<float>();
        case ope::DataType::FLOAT64: return py::dtype::of<double>();
        default: throw BufferError("Unsupported IOBuffer data type");
    }
}

// 1-D view of the buffer's memory; the view's base is the IOBuffer itself
py::array as_numpy(const ope::IOBuffer& b) {
    auto& buf = const_cast<ope::IOBuffer&>(b);
    py::dtype dt = numpy_dtype(buf.getDataType());
    const py::ssize_t n = static_cast<py::ssize_t>(buf.getSizeInBytes() / dt.itemsize());
    return py::array(dt, {n}, {dt.itemsize()}, buf.getDataPointer(), py::cast(&buf, py::return_value_policy::reference));
}

py::array_t<float> copy_out(const float* p, size_t n) {
    py::array_t<float> a(static_cast<py::ssize_t>(n));
    if (n) std::memcpy(a.mutable_data(), p, n * sizeof(float));
    return a;
}

std::vector<float> contiguous_1d(const py::array_t<float, py::array::c_style | py::array::forcecast>& a,
                                 const char* what) {
    if (a.ndim() != 1) throw BufferError(std::string(what) + " must be a 1D array");
    return std::vector<float>(a.data(), a.data() + a.size());
}

class PyProcessor {
public:
    ope::Processor proc;
    py::object single_cb = py::none();
    py::object error_cb = py::none();

    explicit PyProcessor(ope::Backend b) : proc(b) {}

    ~PyProcessor() {
        py::gil_scoped_release nogil;
        proc.cleanup();
    }

    void set_callback(py::function cb, py::object err) {
        single_cb = cb;
        error_cb = err;
        py::gil_scoped_release nogil;
        proc.setOutputCallback([this](const ope::IOBuffer& out) {
            py::gil_scoped_acquire gil;
            try {
                single_cb(as_numpy(out));
            } catch (const std::exception& e) {
                if (!error_cb.is_none()) {
                    try {
                        error_cb(py::str(e.what()));
                    } catch (...) {
                        py::print("Error in error_callback:", e.what());
                    }
                } else {
                    py::print("Error in callback:", e.what());
                }
            }
        });
    }

    ope::Processor::CallbackId add(py::function cb) {
        // the C++ side copies the closure without the GIL: hold the Python
        // function through a shared pointer whose last owner drops it under the GIL
        std::shared_ptr<py::function> fn(new py::function(std::move(cb)), [](py::function* f) {
            py::gil_scoped_acquire gil;
            delete f;
        });
        auto wrapped = [fn](const ope::IOBuffer& out) {
            py::gil_scoped_acquire gil;
            try {
                (*fn)(as_numpy(out));
            } catch (const std::exception& e) {
                py::print("Error in callback:", e.what());
            }
        };
        py::gil_scoped_release nogil;
        return proc.addOutputCallback(std::move(wrapped));
    }

    bool remove(ope::Processor::CallbackId id) {
        py::gil_scoped_release nogil;
        return proc.removeOutputCallback(id);
    }

    void clear() {
        py::gil_scoped_release nogil;
        proc.clearOutputCallbacks();
    }

    void process(py::array view) {
        // walk the .base chain of the view down to the IOBuffer it came from
        py::object o = view;
        ope::IOBuffer* buf = nullptr;
        for (int depth = 0; depth < 8 && !o.is_none(); ++depth) {
            if (py::isinstance<ope::IOBuffer>(o)) {
                buf = o.cast<ope::IOBuffer*>();
                break;
            }
            if (!py::hasattr(o, "base")) break;
            o = o.attr("base");
        }
        if (!buf) throw BufferError("Buffer array is not a view of an IOBuffer. Use get_next_available_buffer() first.");
        py::gil_scoped_release nogil;
        proc.process(*buf);
    }

    py::array next_buffer() {
        ope::IOBuffer* b;
        {
            py::gil_scoped_release nogil;
            b = &proc.getNextAvailableInputBuffer();
        }
        return as_numpy(*b);
    }

    void initialize() {
        try {
            py::gil_scoped_release nogil;
            proc.initialize();
        } catch (const std::exception& e) {
            throw InitializationError(std::string("Initialization failed: ") + e.what());
        }
    }

    void stop() {
        py::gil_scoped_release nogil;
        proc.cleanup();
    }
};

}  // namespace

PYBIND11_MODULE(octproengine, m) {
    m.doc() = "OCTproEngine API on the B200 (sm_100a) processing backend";

    py::register_exception<InitializationError>(m, "InitializationError");
    py::register_exception<ConfigurationError>(m, "ConfigurationError");
    py::register_exception<BufferError>(m, "BufferError");
    py::register_exception<ProcessingError>(m, "ProcessingError");
    py::register_exception<BackendError>(m, "BackendError");

    py::class_<ope::IOBuffer>(m, "IOBuffer", py::module_local())
        .def("get_size", &ope::IOBuffer::getSizeInBytes)
        .def("get_data_type", &ope::IOBuffer::getDataType);

    py::enum_<ope::Backend>(m, "Backend")
        .value("CUDA", ope::Backend::CUDA)
        .value("CPU", ope::Backend::CPU)
        .value("B200", ope::Backend::B200)
        .export_values();

    py::enum_<ope::DataType>(m, "DataType")
        .value("UINT8", ope::DataType::UINT8)
        .value("UINT16", ope::DataType::UINT16)
        .value("UINT32", ope::DataType::UINT32)
        .value("UINT64", ope::DataType::UINT64)
        .value("INT8", ope::DataType::INT8)
        .value("INT16", ope::DataType::INT16)
        .value("INT32", ope::DataType::INT32)
        .value("INT64", ope::DataType::INT64)
        .value("FLOAT32", ope::DataType::FLOAT32)
        .value("FLOAT64", ope::DataType::FLOAT64)
        .value("COMPLEX_FLOAT32", ope::DataType::COMPLEX_FLOAT32)
        .value("COMPLEX_FLOAT64", ope::DataType::COMPLEX_FLOAT64)
        .export_values();

    py::enum_<ope::InterpolationMethod>(m, "InterpolationMethod")
        .value("LINEAR", ope::InterpolationMethod::LINEAR)
        .value("CUBIC", ope::InterpolationMethod::CUBIC)
        .value("LANCZOS", ope::InterpolationMethod::LANCZOS)
        .export_values();

    py::enum_<ope::WindowType>(m, "WindowType")
        .value("HANN", ope::WindowType::HANN)
        .value("GAUSS", ope::WindowType::GAUSS)
        .value("SINE", ope::WindowType::SINE)
        .value("LANCZOS", ope::WindowType::LANCZOS)
        .value("RECTANGULAR", ope::WindowType::RECTANGULAR)
        .value("FLAT_TOP", ope::WindowType::FLAT_TOP)
        .export_values();

    using PC = ope::ProcessorConfiguration;
    auto coeff_get = [](const float* c) { return std::vector<float>(c, c + 4); };
    auto coeff_set = [](float* dst, const std::vector<float>& v) {
        if (v.size() != 4) throw std::runtime_error("Coefficients must have exactly 4 elements");
        std::copy(v.begin(), v.end(), dst);
    };

    py::class_<PC::DataParameters>(m, "DataParameters")
        .def(py::init<>())
        .def_readwrite("signal_length", &PC::DataParameters::signalLength)
        .def_readwrite("samples_per_buffer", &PC::DataParameters::samplesPerBuffer)
        .def_readwrite("ascans_per_bscan", &PC::DataParameters::ascansPerBscan)
        .def_readwrite("bscans_per_buffer", &PC::DataParameters::bscansPerBuffer)
        .def_readwrite("input_data_type", &PC::DataParameters::inputDataType)
        .def_readwrite("bitshift", &PC::DataParameters::bitshift)
        .def("get_bit_depth", &PC::DataParameters::getBitDepth)
        .def("get_bytes_per_sample", &PC::DataParameters::getBytesPerSample);

    py::class_<PC::ProcessingParameters>(m, "ProcessingParameters")
        .def(py::init<>())
        .def_readwrite("n_streams", &PC::ProcessingParameters::nStreams)
        .def_readwrite("n_buffers", &PC::ProcessingParameters::nBuffers)
        .def_readwrite("grid_size", &PC::ProcessingParameters::gridSize)
        .def_readwrite("block_size", &PC::ProcessingParameters::blockSize);

    py::class_<PC::ResamplingParameters>(m, "ResamplingParameters")
        .def(py::init<>())
        .def_readwrite("enabled", &PC::ResamplingParameters::enabled)
        .def_readwrite("interpolation_method", &PC::ResamplingParameters::interpolationMethod)
        .def_readwrite("use_coefficients", &PC::ResamplingParameters::useCoefficients)
        .def_property(
            "coefficients", [=](const PC::ResamplingParameters& s) { return coeff_get(s.coefficients); },
            [=](PC::ResamplingParameters& s, const std::vector<float>& v) { coeff_set(s.coefficients, v); })
        .def_readwrite("use_custom_curve", &PC::ResamplingParameters::useCustomCurve);

    py::class_<PC::WindowingParameters>(m, "WindowingParameters")
        .def(py::init<>())
        .def_readwrite("enabled", &PC::WindowingParameters::enabled)
        .def_readwrite("window_type", &PC::WindowingParameters::windowType)
        .def_readwrite("window_center_position", &PC::WindowingParameters::windowCenterPosition)
        .def_readwrite("window_fill_factor", &PC::WindowingParameters::windowFillFactor)
        .def_readwrite("use_custom_curve", &PC::WindowingParameters::useCustomCurve);

    py::class_<PC::DispersionCompensationParameters>(m, "DispersionCompensationParameters")
        .def(py::init<>())
        .def_readwrite("enabled", &PC::DispersionCompensationParameters::enabled)
        .def_readwrite("use_coefficients", &PC::DispersionCompensationParameters::useCoefficients)
        .def_property(
            "coefficients", [=](const PC::DispersionCompensationParameters& s) { return coeff_get(s.coefficients); },
            [=](PC::DispersionCompensationParameters& s, const std::vector<float>& v) { coeff_set(s.coefficients, v); })
        .def_readwrite("factor", &PC::DispersionCompensationParameters::factor)
        .def_readwrite("use_custom_curve", &PC::DispersionCompensationParameters::useCustomCurve);

    py::class_<PC::BackgroundRemovalParameters>(m, "BackgroundRemovalParameters")
        .def(py::init<>())
        .def_readwrite("enabled", &PC::BackgroundRemovalParameters::enabled)
        .def_readwrite("rolling_average_window_size", &PC::BackgroundRemovalParameters::rollingAverageWindowSize);

    py::class_<PC::PostProcessingParameters>(m, "PostProcessingParameters")
        .def(py::init<>())
        .def_readwrite("background_removal", &PC::PostProcessingParameters::backgroundRemoval)
        .def_readwrite("background_weight", &PC::PostProcessingParameters::backgroundWeight)
        .def_readwrite("background_offset", &PC::PostProcessingParameters::backgroundOffset)
        .def_readwrite("log_scaling", &PC::PostProcessingParameters::logScaling)
        .def_readwrite("grayscale_max", &PC::PostProcessingParameters::grayscaleMax)
        .def_readwrite("grayscale_min", &PC::PostProcessingParameters::grayscaleMin)
        .def_readwrite("addend", &PC::PostProcessingParameters::addend)
        .def_readwrite("multiplicator", &PC::PostProcessingParameters::multiplicator)
        .def_readwrite("bscan_flip", &PC::PostProcessingParameters::bscanFlip)
        .def_readwrite("sinusoidal_scan_correction", &PC::PostProcessingParameters::sinusoidalScanCorrection)
        .def_readwrite("fixed_pattern_noise_removal", &PC::PostProcessingParameters::fixedPatternNoiseRemoval)
        .def_readwrite("fixed_pattern_noise_bscan_count", &PC::PostProcessingParameters::fixedPatternNoiseBscanCount)
        .def_readwrite("continuous_fixed_pattern_noise_determination",
                       &PC::PostProcessingParameters::continuousFixedPatternNoiseDetermination);

    auto curve_or_empty = [](bool has, const float* p, size_t n) {
        return has ? copy_out(p, n) : py::array_t<float>(0);
    };
    py::class_<PC>(m, "ProcessorConfiguration")
        .def(py::init<>())
        .def_readwrite("data", &PC::dataParams)
        .def_readwrite("processing", &PC::processingParams)
        .def_readwrite("resampling", &PC::resamplingParams)
        .def_readwrite("windowing", &PC::windowingParams)
        .def_readwrite("dispersion", &PC::dispersionParams)
        .def_readwrite("background_removal", &PC::backgroundRemovalParams)
        .def_readwrite("post_processing", &PC::postProcessingParams)
        .def("set_custom_resampling_curve",
             [](PC& s, py::array_t<float, py::array::c_style | py::array::forcecast> c) {
                 auto v = contiguous_1d(c, "Resampling curve");
                 s.setCustomResamplingCurve(v.data(), v.size());
             })
        .def("set_custom_window_curve",
             [](PC& s, py::array_t<float, py::array::c_style | py::array::forcecast> c) {
                 auto v = contiguous_1d(c, "Window curve");
                 s.setCustomWindowCurve(v.data(), v.size());
             })
        .def("set_custom_dispersion_curve",
             [](PC& s, py::array_t<float, py::array::c_style | py::array::forcecast> c) {
                 auto v = contiguous_1d(c, "Dispersion curve");
                 s.setCustomDispersionCurve(v.data(), v.size());
             })
        .def("get_custom_resampling_curve",
             [=](const PC& s) {
                 return curve_or_empty(s.hasCustomResamplingCurve(), s.getCustomResamplingCurve(),
                                       s.getCustomResamplingCurveSize());
             })
        .def("get_custom_window_curve",
             [=](const PC& s) {
                 return curve_or_empty(s.hasCustomWindowCurve(), s.getCustomWindowCurve(), s.getCustomWindowCurveSize());
             })
        .def("get_custom_dispersion_curve",
             [=](const PC& s) {
                 return curve_or_empty(s.hasCustomDispersionCurve(), s.getCustomDispersionCurve(),
                                       s.getCustomDispersionCurveSize());
             })
        .def("has_custom_resampling_curve", &PC::hasCustomResamplingCurve)
        .def("has_custom_window_curve", &PC::hasCustomWindowCurve)
        .def("has_custom_dispersion_curve", &PC::hasCustomDispersionCurve)
        .def("save_to_file", &PC::saveToFile)
        .def("load_from_file", &PC::loadFromFile)
        .def("validate", &PC::validate);

    using P = PyProcessor;
    using F1 = py::array_t<float, py::array::c_style | py::array::forcecast>;
    py::class_<P>(m, "Processor")
        .def(py::init<ope::Backend>(), py::arg("backend") = ope::Backend::CUDA)
        .def("initialize", &P::initialize)
        .def("stop", &P::stop)
        .def("load_config",
             [](P& s, const std::string& f) {
                 try {
                     s.proc.loadConfigurationFromFile(f);
                 } catch (const std::exception& e) {
                     throw ConfigurationError(std::string("Failed to load config: ") + e.what());
                 }
             },
             py::arg("filepath"))
        .def("save_config",
             [](const P& s, const std::string& f) {
                 try {
                     s.proc.saveConfigurationToFile(f);
                 } catch (const std::exception& e) {
                     throw ConfigurationError(std::string("Failed to save config: ") + e.what());
                 }
             },
             py::arg("filepath"))
        .def_property_readonly("config", [](const P& s) { return s.proc.getConfig(); })
        .def("set_config",
             [](P& s, const PC& c) {
                 py::gil_scoped_release nogil;
                 s.proc.setConfig(c);
             },
             py::arg("config"))
        .def("set_input_parameters",
             [](P& s, int n, int a, int b, ope::DataType t) { s.proc.setInputParameters(n, a, b, t); },
             py::arg("samples_per_ascan"), py::arg("ascans_per_bscan"), py::arg("bscans_per_buffer"),
             py::arg("data_type"))
        .def("set_backend",
             [](P& s, ope::Backend b) {
                 py::gil_scoped_release nogil;
                 s.proc.setBackend(b);
             },
             py::arg("backend"))
        .def("get_backend", [](const P& s) { return s.proc.getBackend(); })
        .def("set_callback", &P::set_callback, py::arg("callback"), py::arg("error_callback") = py::none())
        .def("add_output_callback", &P::add, py::arg("callback"))
        .def("remove_output_callback", &P::remove, py::arg("callback_id"))
        .def("clear_output_callbacks", &P::clear)
        .def("get_callback_count", [](const P& s) { return s.proc.getCallbackCount(); })
        .def("process", &P::process, py::arg("buffer"))
        .def("get_next_available_buffer", &P::next_buffer)
        // resampling
        .def("set_resampling_coefficients",
             [](P& s, const std::array<float, 4>& c) { s.proc.setResamplingCoefficients(c.data()); },
             py::arg("coefficients"))
        .def("set_custom_resampling_curve",
             [](P& s, F1 c) {
                 auto v = contiguous_1d(c, "Resampling curve");
                 s.proc.setCustomResamplingCurve(v.data(), v.size());
             },
             py::arg("curve"))
        .def("use_custom_resampling_curve", [](P& s, bool u) { s.proc.useCustomResamplingCurve(u); },
             py::arg("use_custom"))
        .def("enable_resampling", [](P& s, bool e) { s.proc.enableResampling(e); }, py::arg("enable"))
        .def("set_interpolation_method", [](P& s, ope::InterpolationMethod i) { s.proc.setInterpolationMethod(i); },
             py::arg("method"))
        // dispersion
        .def("set_dispersion_coefficients",
             [](P& s, const std::array<float, 4>& c, float f) { s.proc.setDispersionCoefficients(c.data(), f); },
             py::arg("coefficients"), py::arg("factor") = 1.0f)
        .def("set_custom_dispersion_curve",
             [](P& s, F1 c) {
                 auto v = contiguous_1d(c, "Dispersion curve");
                 s.proc.setCustomDispersionCurve(v.data(), v.size());
             },
             py::arg("curve"))
        .def("use_custom_dispersion_curve", [](P& s, bool u) { s.proc.useCustomDispersionCurve(u); },
             py::arg("use_custom"))
        .def("enable_dispersion_compensation", [](P& s, bool e) { s.proc.enableDispersionCompensation(e); },
             py::arg("enable"))
        // windowing
        .def("set_window_parameters",
             [](P& s, ope::WindowType t, float c, float f) { s.proc.setWindowParameters(t, c, f); },
             py::arg("window_type"), py::arg("center"), py::arg("fill_factor"))
        .def("set_custom_window_curve",
             [](P& s, F1 c) {
                 auto v = contiguous_1d(c, "Window curve");
                 s.proc.setCustomWindowCurve(v.data(), v.size());
             },
             py::arg("curve"))
        .def("use_custom_window_curve", [](P& s, bool u) { s.proc.useCustomWindowCurve(u); }, py::arg("use_custom"))
        .def("enable_windowing", [](P& s, bool e) { s.proc.enableWindowing(e); }, py::arg("enable"))
        // post-processing
        .def("set_grayscale_range", [](P& s, float lo, float hi) { s.proc.setGrayscaleRange(lo, hi); },
             py::arg("min"), py::arg("max"))
        .def("set_signal_multiplicator_and_addend",
             [](P& s, float mul, float add) { s.proc.setSignalMultiplicatorAndAddend(mul, add); },
             py::arg("multiplicator"), py::arg("addend"))
        .def("enable_log_scaling", [](P& s, bool e) { s.proc.enableLogScaling(e); }, py::arg("enable"))
        .def("enable_background_removal", [](P& s, bool e) { s.proc.enableBackgroundRemoval(e); }, py::arg("enable"))
        .def("set_background_removal_window_size", [](P& s, int w) { s.proc.setBackgroundRemovalWindowSize(w); },
             py::arg("window_size"))
        .def("enable_bscan_flip", [](P& s, bool e) { s.proc.enableBscanFlip(e); }, py::arg("enable"))
        .def("enable_sinusoidal_scan_correction", [](P& s, bool e) { s.proc.enableSinusoidalScanCorrection(e); },
             py::arg("enable"))
        .def("enable_fixed_pattern_noise_removal", [](P& s, bool e) { s.proc.enableFixedPatternNoiseRemoval(e); },
             py::arg("enable"))
        .def("enable_post_process_background_subtraction",
             [](P& s, bool e) { s.proc.enablePostProcessBackgroundSubtraction(e); }, py::arg("enable"))
        // post-process background profile
        .def("request_post_process_background_recording",
             [](P& s) {
                 py::gil_scoped_release nogil;
                 s.proc.requestPostProcessBackgroundRecording();
             })
        .def("set_post_process_background_weight", [](P& s, float w) { s.proc.setPostProcessBackgroundWeight(w); },
             py::arg("weight"))
        .def("set_post_process_background_offset", [](P& s, float o) { s.proc.setPostProcessBackgroundOffset(o); },
             py::arg("offset"))
        .def("has_post_process_background_profile",
             [](const P& s) { return s.proc.hasPostProcessBackgroundProfile(); })
        .def("get_post_process_background_profile_size",
             [](const P& s) { return s.proc.getPostProcessBackgroundProfileSize(); })
        .def("get_post_process_background_profile",
             [](const P& s) {
                 if (!s.proc.hasPostProcessBackgroundProfile()) throw BufferError("No background profile available");
                 return copy_out(s.proc.getPostProcessBackgroundProfile(), s.proc.getPostProcessBackgroundProfileSize());
             })
        .def("set_post_process_background_profile",
             [](P& s, F1 p) {
                 auto v = contiguous_1d(p, "Background profile");
                 s.proc.setPostProcessBackgroundProfile(v.data(), v.size());
             },
             py::arg("profile"))
        .def("save_post_process_background_profile_to_file",
             [](const P& s, const std::string& f) {
                 try {
                     s.proc.savePostProcessBackgroundProfileToFile(f);
                 } catch (const std::exception& e) {
                     throw ConfigurationError(std::string("Failed to save background profile: ") + e.what());
                 }
             },
             py::arg("filepath"))
        .def("load_post_process_background_profile_from_file",
             [](P& s, const std::string& f) {
                 try {
                     s.proc.loadPostProcessBackgroundProfileFromFile(f);
                 } catch (const std::exception& e) {
                     throw ConfigurationError(std::string("Failed to load background profile: ") + e.what());
                 }
             },
             py::arg("filepath"))
        // fixed-pattern noise
        .def("request_fixed_pattern_noise_determination",
             [](P& s) {
                 py::gil_scoped_release nogil;
                 s.proc.requestFixedPatternNoiseDetermination();
             })
        .def("enable_continuous_fixed_pattern_noise_determination",
             [](P& s, bool e) { s.proc.enableContinuousFixedPatternNoiseDetermination(e); }, py::arg("enable"))
        .def("set_fixed_pattern_noise_bscan_count", [](P& s, int n) { s.proc.setFixedPatternNoiseBscanCount(n); },
             py::arg("length"))
        .def("has_fixed_pattern_noise_profile", [](const P& s) { return s.proc.hasFixedPatternNoiseProfile(); })
        .def("get_fixed_pattern_noise_profile_size",
             [](const P& s) { return s.proc.getFixedPatternNoiseProfileSize(); })
        .def("get_fixed_pattern_noise_profile",
             [](const P& s) {
                 if (!s.proc.hasFixedPatternNoiseProfile())
                     throw BufferError("No fixed-pattern noise profile available");
                 return copy_out(s.proc.getFixedPatternNoiseProfile(), 2 * s.proc.getFixedPatternNoiseProfileSize());
             })
        .def("set_fixed_pattern_noise_profile",
             [](P& s, F1 p) {
                 auto v = contiguous_1d(p, "fixed-pattern noise profile");
                 if (v.size() % 2)
                     throw BufferError(
                         "fixed-pattern noise profile must have even length (interleaved real/imag pairs)");
                 s.proc.setFixedPatternNoiseProfile(v.data(), v.size() / 2);
             },
             py::arg("profile"))
        .def("save_fixed_pattern_noise_profile_to_file",
             [](const P& s, const std::string& f) {
                 try {
                     s.proc.saveFixedPatternNoiseProfileToFile(f);
                 } catch (const std::exception& e) {
                     throw ConfigurationError(std::string("Failed to save fixed-pattern noise profile: ") + e.what());
                 }
             },
             py::arg("filepath"))
        .def("load_fixed_pattern_noise_profile_from_file",
             [](P& s, const std::string& f) {
                 try {
                     s.proc.loadFixedPatternNoiseProfileFromFile(f);
                 } catch (const std::exception& e) {
                     throw ConfigurationError(std::string("Failed to load fixed-pattern noise profile: ") + e.what());
                 }
             },
             py::arg("filepath"))
        .def("__enter__", [](P& s) -> P& { return s; }, py::return_value_policy::reference)
        .def("__exit__", [](P& s, py::object, py::object, py::object) { s.stop(); })
        .def("__repr__", [](const P& s) {
            const auto b = s.proc.getBackend();
            return std::string("<Processor(backend=") +
                   (b == ope::Backend::CPU ? "CPU" : b == ope::Backend::CUDA ? "CUDA" : "B200") + ")>";
        });

    m.attr("__version__") = "1.0.0+b200";
}
