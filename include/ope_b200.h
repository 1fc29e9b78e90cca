/*
 * ope_b200.h -- C ABI of the B200 (sm_100a) backend for the OCTproEngine
 * per-A-scan processing chain.
 *
 * This is the drop-in boundary. The reference dispatches the chain through the
 * abstract C++ class ope::ProcessingBackend (src/backends/backend_interface.h:12-165),
 * selected by ope::Backend in Processor::Impl::createBackend
 * (src/core/processor.cpp:38-50). Every entry point below replaces one method
 * of that interface (cited per declaration) with a plain-C call: opaque
 * handle, plain pointers and sizes, integer status codes. No C++ or torch type
 * crosses this boundary. The C++ class ope::B200Backend (octproengine_b200/host)
 * wraps these calls and turns a non-zero status into std::runtime_error /
 * std::invalid_argument, the reference's error convention
 * (src/backends/cuda/cuda_backend.cu:14-33, src/core/processor.cpp:136-138).
 *
 * Numeric conventions follow the reference:
 *   - input sample types are ope::DataType values (include/types.h:6-19);
 *   - interpolation and window types are ope::InterpolationMethod /
 *     ope::WindowType values (include/processorconfiguration.h:16-29);
 *   - a buffer is bscans x ascans x samples, A-scans contiguous; the output is
 *     bscans x ascans x (samples/2) float32;
 *   - the dispersion curve handed to the backend is 2*N interleaved
 *     (cos, sin) floats, resampling and window curves are N floats.
 *
 * Thread safety: one context may be used from one thread at a time, except
 * ope_b200_submit / ope_b200_wait / ope_b200_ring_* which are safe between a
 * producer and a consumer thread.
 */
#ifndef OPE_B200_H
#define OPE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define OPE_B200_API __attribute__((visibility("default")))
#else
#define OPE_B200_API
#endif

#define OPE_B200_ABI_VERSION 1

/* Status codes. */
#define OPE_B200_OK 0
#define OPE_B200_E_INVALID (-1)     /* bad argument or configuration */
#define OPE_B200_E_UNSUPPORTED (-2) /* valid for the reference, not supported here */
#define OPE_B200_E_CUDA (-3)        /* CUDA runtime error */
#define OPE_B200_E_TIMEOUT (-4)     /* a bounded wait expired */
#define OPE_B200_E_STATE (-5)       /* call not valid in the current state */
#define OPE_B200_E_NOMEM (-6)       /* allocation failed */
#define OPE_B200_E_DEVICE (-7)      /* a kernel reported an error status */

/* Subset of ope::ProcessorConfiguration (include/processorconfiguration.h:31-180)
 * the chain reads. Enum-valued fields carry the reference enum values. */
typedef struct ope_b200_config {
    int32_t signal_length;     /* DataParameters::signalLength (N)            */
    int32_t ascans_per_bscan;  /* DataParameters::ascansPerBscan (A)          */
    int32_t bscans_per_buffer; /* DataParameters::bscansPerBuffer (B)         */
    int32_t input_dtype;       /* DataParameters::inputDataType (ope::DataType) */
    int32_t bitshift;          /* DataParameters::bitshift: 8/16-bit samples >> 4 (the reference
                                  CUDA backend's rule); ignored for 32-bit samples */
    int32_t resampling_enabled;
    int32_t interpolation; /* ope::InterpolationMethod */
    int32_t windowing_enabled;
    int32_t dispersion_enabled;
    int32_t dc_removal_enabled; /* BackgroundRemovalParameters::enabled          */
    int32_t dc_window;          /* BackgroundRemovalParameters::rollingAverageWindowSize */
    int32_t log_scaling;
    float grayscale_min;
    float grayscale_max;
    float addend;
    float multiplicator;
    int32_t fpn_removal;     /* PostProcessingParameters::fixedPatternNoiseRemoval */
    int32_t fpn_bscan_count; /* ::fixedPatternNoiseBscanCount                  */
    int32_t fpn_continuous;  /* ::continuousFixedPatternNoiseDetermination     */
    int32_t post_bg_removal; /* PostProcessingParameters::backgroundRemoval    */
    float bg_weight;
    float bg_offset;
    int32_t bscan_flip;
    int32_t sinusoidal_correction;
    int32_t float32_as_uint32; /* 1: read FLOAT32 input as uint32 like the reference
                                  backends do (cpu_kernels.tpp:47-52); 0: as float */
    int32_t device;            /* CUDA device ordinal                           */
    int32_t num_input_buffers; /* host input ring depth (>= 2)                  */
    int32_t dc_split;          /* 1 (default): exact DC split -- each A-scan's integer
                                  mean is subtracted before the chain and its float64
                                  response added back after the DFT (same quantity,
                                  lower float32 error; ignored with DC removal on) */
    int32_t dc_reference_order; /* rolling-average DC removal: 0 (default) = exact integer
                                  window sums; 1 = the reference CPU backend's sequential
                                  float prefix sum (rollingAverageDCRemoval,
                                  cpu_kernels.tpp:56-82), bit for bit */
    int32_t reserved[7];
} ope_b200_config;

typedef struct ope_b200_ctx ope_b200_ctx;

/* Fills `cfg` with the reference defaults (processorconfiguration.h:49-171). */
OPE_B200_API void ope_b200_config_default(ope_b200_config* cfg);

/* ---- lifecycle: ProcessingBackend::initialize / cleanup (backend_interface.h:17-18) ---- */
OPE_B200_API int ope_b200_create(const ope_b200_config* cfg, ope_b200_ctx** out);
OPE_B200_API void ope_b200_destroy(ope_b200_ctx* ctx);
/* ProcessingBackend::updateConfig (backend_interface.h:27): non-dimension fields only. */
OPE_B200_API int ope_b200_update_config(ope_b200_ctx* ctx, const ope_b200_config* cfg);
/* Last error message of this context (never NULL); with ctx == NULL, why the calling
 * thread's last ope_b200_create failed. */
OPE_B200_API const char* ope_b200_last_error(const ope_b200_ctx* ctx);

/* ---- hot-swap curves: ProcessingBackend::update{Resampling,Dispersion,Window}Curve
 *      (backend_interface.h:30-32). Copied; the caller keeps ownership.  Updates are
 *      ordered after all work already enqueued on the context. ---- */
OPE_B200_API int ope_b200_set_resampling_curve(ope_b200_ctx* ctx, const float* curve, size_t n);
OPE_B200_API int ope_b200_set_dispersion_curve(ope_b200_ctx* ctx, const float* cos_sin, size_t n_floats);
OPE_B200_API int ope_b200_set_window_curve(ope_b200_ctx* ctx, const float* curve, size_t n);

/* ---- processing: ProcessingBackend::process (backend_interface.h:24) ---- */
/* Device-resident: d_in holds A*B raw A-scans (16-byte aligned), d_out
 * receives A*B*(N/2) floats. Asynchronous on `stream` (a cudaStream_t; NULL is
 * the CUDA default stream). */
OPE_B200_API int ope_b200_process_device(ope_b200_ctx* ctx, const void* d_in, float* d_out, void* stream);
/* Same for an explicit A-scan count (any count >= 1), for callers that batch. */
OPE_B200_API int ope_b200_process_device_n(ope_b200_ctx* ctx, const void* d_in, float* d_out, int64_t num_ascans,
                                           void* stream);
/* Complex output: the chain up to the inverse DFT (after the fixed-pattern
 * subtraction, before magnitude/log), bins [0, N/2) of each A-scan as
 * interleaved (re, im) float pairs -- num_ascans * (N/2) * 8 bytes at d_bins
 * (8-byte aligned). Replaces the complex stage the reference keeps in
 * allIfftOutputs (cpu_backend.cpp:231-242); used by autofocus and by tests. */
OPE_B200_API int ope_b200_process_bins_device(ope_b200_ctx* ctx, const void* d_in, void* d_bins, int64_t num_ascans,
                                              void* stream);
/* Host to host, synchronous: copies h_in to the device, runs the chain, copies
 * the result to h_out and waits. */
OPE_B200_API int ope_b200_process_host(ope_b200_ctx* ctx, const void* h_in, float* h_out);

/* ---- streaming ring: the IOBuffer path of ProcessingBackend::process and
 *      getNextAvailableInputBuffer (backend_interface.h:24,35-37).
 *      Depth = num_input_buffers (>= 2). A frame is copied in, processed and
 *      copied out on its own stream; neighbouring frames overlap. ---- */
OPE_B200_API int ope_b200_ring_depth(ope_b200_ctx* ctx);
/* Page-locks caller memory so copies from it are asynchronous (IOBuffers). */
OPE_B200_API int ope_b200_host_register(void* ptr, size_t bytes);
OPE_B200_API int ope_b200_host_unregister(void* ptr);
/* Enqueues one buffer (A*B A-scans at h_in); returns a ticket. Fails with
 * OPE_B200_E_STATE when every slot still holds an unreleased frame. */
OPE_B200_API int ope_b200_submit(ope_b200_ctx* ctx, const void* h_in, uint64_t* ticket);
/* Same, with the output copied into the caller's buffer h_out (A*B*(N/2)
 * floats; page-locked for an asynchronous copy) instead of the slot's own. */
OPE_B200_API int ope_b200_submit_to(ope_b200_ctx* ctx, const void* h_in, float* h_out, uint64_t* ticket);
/* Waits until h_in of `ticket` has been copied to the device (the caller may
 * then reuse it); timeout_ms < 0 waits without limit. */
OPE_B200_API int ope_b200_input_released(ope_b200_ctx* ctx, uint64_t ticket, int32_t timeout_ms);
/* The device copy of a submitted frame's input (its ring slot), for more work
 * on the same data on another stream (a per-chunk dispersion fit) without a
 * second transfer: makes `stream` wait for the frame's input copy and returns
 * the slot's device address. Valid until ope_b200_release(ticket); work that
 * reads it must have finished by then (the slot takes a later frame). */
OPE_B200_API int ope_b200_frame_device_input(ope_b200_ctx* ctx, uint64_t ticket, void* stream, const void** d_in);
/* Waits for the frame; *h_out points at its A*B*(N/2) floats in pinned host
 * memory, valid until ope_b200_release(ticket). */
OPE_B200_API int ope_b200_wait(ope_b200_ctx* ctx, uint64_t ticket, int32_t timeout_ms, const float** h_out);
OPE_B200_API int ope_b200_release(ope_b200_ctx* ctx, uint64_t ticket);

/* ---- fixed-pattern noise: ProcessingBackend::{request,set,get}FixedPatternNoise*
 *      (backend_interface.h:45-47). Profiles are interleaved (re, im) pairs. ---- */
OPE_B200_API int ope_b200_request_fpn_determination(ope_b200_ctx* ctx);
OPE_B200_API int ope_b200_set_fpn_profile(ope_b200_ctx* ctx, const float* interleaved, size_t complex_pairs);
OPE_B200_API int ope_b200_get_fpn_profile(ope_b200_ctx* ctx, float* out, size_t cap_pairs, size_t* pairs);

/* Fixed-pattern-noise determination that allocates nothing. No counterpart in
 * the reference. For callers that may not allocate device memory once running:
 * a real-time acquisition thread must not stall on cudaMalloc/cudaFree (they
 * can synchronise the whole device), and integrations that budget all device
 * memory at start-up may not allocate afterwards. The allocating path
 * (request + process) grows a scratch buffer with cudaMalloc on first use; this
 * call keeps its scratch in one static device array of 3.4 MiB, which every
 * GPU that loads the library holds until the process exits.
 *
 * Computes the minimum-variance-mean profile (cpu_kernels.tpp:402-458) of the
 * first fpn_bscan_count * ascans_per_bscan A-scans of the device buffer d_in
 * (num_ascans A-scans, at least that many) and writes N/2 interleaved
 * (re, im) float pairs to d_profile (8-byte aligned). Asynchronous on
 * `stream`; the context's own FPN state is not changed. Limits: signal length
 * up to 4096 (OPE_B200_E_UNSUPPORTED beyond). Every call looks up the array's
 * device address in the current context (no cached address survives a device
 * reset); make the first call on a device before any stream capture. All calls
 * share the one array: calls that overlap on the GPU race and corrupt each
 * other's results. The call blocks the host in one case: when a curve or the
 * configuration changed since the last processing call, it first rebuilds the
 * context's device tables (a synchronous upload). A real-time loop avoids that
 * stall by processing one buffer (or calling this once) after every curve or
 * configuration change, before it enters the loop. */
OPE_B200_API int ope_b200_determine_fpn_noalloc(ope_b200_ctx* ctx, const void* d_in, int64_t num_ascans,
                                                float* d_profile, void* stream);

/* ---- post-process background: ProcessingBackend::requestPostProcessBackgroundRecording /
 *      set/getPostProcessBackgroundProfile (backend_interface.h:40-42) ---- */
OPE_B200_API int ope_b200_request_bg_recording(ope_b200_ctx* ctx);
OPE_B200_API int ope_b200_set_bg_profile(ope_b200_ctx* ctx, const float* profile, size_t n);
OPE_B200_API int ope_b200_get_bg_profile(ope_b200_ctx* ctx, float* out, size_t cap, size_t* n);

/* Waits for all work of the context, then reads and clears the device status
 * word (0 = no kernel reported an error). */
OPE_B200_API int ope_b200_synchronize(ope_b200_ctx* ctx, int32_t* device_status);

/* ---- curve generators: ProcessorConfiguration::generate{Resampling,Dispersion,Window}Curve
 *      (src/core/processorconfiguration.cpp:438-589) and the phase -> (cos, sin)
 *      hand-off of Processor::Impl::getDispersionCurve (src/core/processor.cpp:77-99).
 *      Bit-identical to the reference on x86-64. ---- */
OPE_B200_API int ope_b200_generate_resampling_curve(int32_t n, const float coeffs[4], float* out);
OPE_B200_API int ope_b200_generate_dispersion_phase(int32_t n, const float coeffs[4], float* out);
OPE_B200_API int ope_b200_generate_window_curve(int32_t n, int32_t window_type, float center, float fill,
                                                float* out);
OPE_B200_API int ope_b200_phase_to_cos_sin(const float* phase, size_t n, float* out_interleaved);

/* ---- differentiable chain for autofocus. No counterpart in the reference (its
 *      dispersion and k-mapping coefficients are set by hand or swept,
 *      processor.cpp:371-470); the forward follows the chain of
 *      CpuBackend::Impl::processData (cpu_backend.cpp:184-264). ----
 *
 * Parameters live in DEVICE memory as float[8]: the dispersion polynomial
 * d0..d3 and the resampling polynomial c0..c3, both in the convention of
 * ProcessorConfiguration::generate{Dispersion,Resampling}Curve
 * (processorconfiguration.cpp:438-482). Every call rebuilds the resampling and
 * window-phase tables on the device from them, so a parameter update needs no
 * host round trip. Each A-scan's integer mean is subtracted before the chain
 * and not added back (the image without its DC term). One handle serves one
 * stream at a time: its tables and partial sums are shared by its calls. */
typedef struct ope_b200_af ope_b200_af;
#define OPE_B200_AF_OUT_INTENSITY 1 /* I = |X|^2, bins [0, N/2)            */
#define OPE_B200_AF_OUT_DB 2        /* 10 log10(I / (N/2)), the reference's log
                                       scale before the grayscale affine map   */
/* n in {1024, 2048, 4096}; input_dtype an ope::DataType (UINT8, UINT16, FLOAT32
 * -- read as float); interpolation an ope::InterpolationMethod; window: N host
 * floats (NULL = rectangular), copied. */
OPE_B200_API int ope_b200_af_create(int32_t n, int32_t input_dtype, int32_t interpolation, const float* window,
                                    int32_t device, ope_b200_af** out);
OPE_B200_API void ope_b200_af_destroy(ope_b200_af* af);
/* DataParameters::bitshift for the fit's data: with `on`, every 8- or 16-bit
 * sample is shifted right by 4 before the chain, in the forward and the
 * adjoint alike, as the processing chain does with the flag set, so a fit
 * sharpens the image the chain will produce. Ignored for float32 input. */
OPE_B200_API int ope_b200_af_set_bitshift(ope_b200_af* af, int32_t on);
OPE_B200_API const char* ope_b200_af_last_error(const ope_b200_af* af);
/* Forward over num_ascans A-scans at d_in (16-byte aligned). d_out (may be
 * NULL): num_ascans x N/2 floats in `output_mode`. d_hs (may be NULL): two
 * doubles, the Shannon entropy H = -sum p ln p of the normalised intensity
 * p = I / S over every bin of every A-scan, and S = sum I. */
OPE_B200_API int ope_b200_af_forward(ope_b200_af* af, const void* d_in, int64_t num_ascans, const float* d_params,
                                     int32_t output_mode, float* d_out, double* d_hs, void* stream);
/* Adjoint: writes dL/dparams (float[8], device) for L = sum(d_grad_out * out)
 * when d_grad_out (num_ascans x N/2, gradient of the `output_mode` output) is
 * given, else for L = H using d_hs from ope_b200_af_forward with the same
 * parameters. Recomputes the forward (nothing is stored between the calls). */
OPE_B200_API int ope_b200_af_backward(ope_b200_af* af, const void* d_in, int64_t num_ascans, const float* d_params,
                                      int32_t output_mode, const float* d_grad_out, const double* d_hs,
                                      float* d_grad_params, void* stream);
/* Same as ope_b200_af_backward for the dispersion coefficients d0..d3 only
 * (entries 4..7, the k-map, are written as 0): the adjoint keeps the resampled
 * samples instead of differentiating the interpolation, which a dispersion
 * fit does not need. Called after ope_b200_af_forward on the same stream with
 * the same d_params pointer, it reuses the device tables that forward built
 * (the values behind d_params must not change between the two calls). */
OPE_B200_API int ope_b200_af_backward_dispersion(ope_b200_af* af, const void* d_in, int64_t num_ascans,
                                                 const float* d_params, int32_t output_mode,
                                                 const float* d_grad_out, const double* d_hs,
                                                 float* d_grad_params, void* stream);
/* 1 when kernels can use `ptr` at that address (device memory, or page-locked
 * host memory under unified addressing), else 0. */
OPE_B200_API int ope_b200_af_kernel_accessible(const void* ptr);
/* Copies `bytes` (<= 4096) on `stream` with one small kernel instead of a
 * copy-engine DMA; both pointers must be kernel-accessible. For a fit's
 * parameters and results, which otherwise wait behind bulk frame copies. */
OPE_B200_API int ope_b200_af_small_copy(void* dst, const void* src, int32_t bytes, void* stream);

/* ---- batched chain: many buffers of uneven geometry in ONE persistent launch.
 *      No counterpart in the reference, whose backends process one IOBuffer of
 *      one geometry per ProcessingBackend::process call (backend_interface.h:24).
 *      Each buffer is described by a configured context (its
 *      ProcessorConfiguration and curves, ope_b200_create + curve setters) and
 *      gets exactly the chain ope_b200_process_device_n runs for it. ----
 *
 * Limits: N in {1024, 2048, 4096}; input UINT8, UINT16 or FLOAT32 (as float);
 * FPN subtraction with a set or determined profile, but no FPN determination
 * (no pending request, no continuous mode). A batch snapshots its contexts'
 * tables at creation: re-create it after changing a context's curves or
 * configuration. One launch of a batch at a time (launches are stream-ordered
 * by the caller; plain launches also wait for the previous one). */
typedef struct ope_b200_batch ope_b200_batch;
typedef struct ope_b200_batch_item {
    ope_b200_ctx* ctx;  /* the buffer's chain configuration               */
    const void* d_in;   /* num_ascans x N raw samples, 16-byte aligned      */
    float* d_out;       /* num_ascans x N/2 floats                          */
    int64_t num_ascans; /* >= 1                                             */
} ope_b200_batch_item;
OPE_B200_API int ope_b200_batch_create(const ope_b200_batch_item* items, int32_t count, ope_b200_batch** out);
OPE_B200_API void ope_b200_batch_destroy(ope_b200_batch* batch);
OPE_B200_API const char* ope_b200_batch_last_error(const ope_b200_batch* batch);
/* One persistent launch over every buffer of the batch, on `stream`. */
OPE_B200_API int ope_b200_batch_run(ope_b200_batch* batch, void* stream);
/* Same launch from a CUDA graph: the first call (and the first after a tuning
 * change) captures it, later calls replay it. The graph keeps the buffer
 * pointers of the batch. */
OPE_B200_API int ope_b200_batch_run_graph(ope_b200_batch* batch, void* stream);
/* Tuning per signal length n: pairs_per_team (pairs of A-scans a team of
 * N/16 threads takes from its length's work counter per grab; the team stages
 * the next pair while computing the current one across grabs and buffers, so
 * the grab size only trades counter traffic against the balance at the end)
 * and radix_schedule, the FFT radix plan: every pass has radix 16 but one
 * short pass (radix N / 16^(passes-1)), run last (0), first (1) or second (2):
 * 1024 = 16*16*4 / 4*16*16 / 16*4*16, 2048 = 16*16*8 / 8*16*16 / 16*8*16;
 * n = 4096 (16*16*16) has only 0. Defaults: 2 and 0. */
OPE_B200_API int ope_b200_batch_set_tuning(ope_b200_batch* batch, int32_t n, int32_t pairs_per_team,
                                           int32_t radix_schedule);
OPE_B200_API int ope_b200_batch_get_tuning(ope_b200_batch* batch, int32_t n, int32_t* pairs_per_team,
                                           int32_t* radix_schedule, float* best_us);
/* Autotuner: for every length in the batch, times each candidate
 * (pairs_per_team in {1, 2, 4, 8} x the radix schedules) on the
 * batch's own buffers of that length (`reps` timed launches each, CUDA
 * events, best kept) and keeps the fastest. Overwrites the outputs. */
OPE_B200_API int ope_b200_batch_autotune(ope_b200_batch* batch, int32_t reps);

/* ---- low-level per-operation API: the unit-level operations of
 *      ProcessingBackend (backend_interface.h:50-164, Processor
 *      include/processor.h:165-282), each one GPU kernel on HOST arrays,
 *      synchronous (copy in, kernel, copy out). Where the reference CPU backend
 *      implements the operation (cpu_backend.cpp:514-733) the arithmetic is its
 *      kernels' (cpu_kernels.tpp); its CUDA backend returns empty results for
 *      all of them (cuda_backend.cu:1133-1296). All outputs are float arrays. ---- */
/* convertInput: samples of bit depth <= 8 / <= 16 / else read as uint8 / uint16 /
 * uint32 and converted to float (cpu_kernels.tpp:24-54; the bitshift flag is not
 * applied, as in the CPU backend). */
OPE_B200_API int ope_b200_op_convert_input(const void* input, int32_t bit_depth, int64_t samples, float* out);
/* kLinearization of one line (method: ope::InterpolationMethod); the first
 * `samples` outputs (cpu_backend.cpp:533-570). */
OPE_B200_API int ope_b200_op_klinearization(const float* input, const float* curve, int32_t method,
                                            int32_t line_width, int64_t samples, float* out);
/* mode 1: windowing (cpu_backend.cpp:572-597); 2: dispersionCompensation, real
 * part, phase as 2*line_width interleaved (cos, sin) (:599-627); 3: dispersion
 * then window (dispersionCompensationAndWindowing). First `samples` outputs. */
OPE_B200_API int ope_b200_op_window_dispersion(const float* input, const float* window, const float* phase_cos_sin,
                                               int32_t mode, int32_t line_width, int64_t samples, float* out);
/* |DFT| of one real line, all line_width outputs: inverse = 1 is the reference's
 * ifft (unnormalised exp(+i), cpu_backend.cpp:634-659), 0 the forward transform
 * (the same magnitudes for a real line). Power-of-two lengths 512..8192 run the
 * chain's own float32 Stockham FFT; other lengths a direct DFT in double. */
OPE_B200_API int ope_b200_op_dft_magnitude(const float* input, int32_t line_width, int32_t inverse, float* out);
/* getMinimumVarianceMean over height rows of width interleaved complex values:
 * 2*width floats (cpu_kernels.tpp:402-458, same double accumulation). */
OPE_B200_API int ope_b200_op_min_variance_mean(const float* input, int32_t width, int32_t height, int32_t segments,
                                               float* out);
/* fixedPatternNoiseRemoval (cpu_backend.cpp:701-733): mean line subtracted as the
 * reference's meanALineSubtraction does on the flattened buffer, then |z|. */
OPE_B200_API int ope_b200_op_fpn_removal(const float* input, const float* mean_line, int32_t line_width,
                                         int32_t num_lines, float* out);
/* rollingAverageBackgroundRemoval per line, the reference kernel's float running
 * sum (cpu_kernels.tpp:56-82). */
OPE_B200_API int ope_b200_op_rolling_dc_removal(const float* input, int32_t window, int32_t line_width,
                                                int32_t num_lines, float* out);
/* bscanFlip with the chain's rule (even B-scans that have a successor mirrored). */
OPE_B200_API int ope_b200_op_bscan_flip(const float* input, int32_t line_width, int32_t lines_per_bscan,
                                        int32_t num_bscans, float* out);
/* sinusoidalScanCorrection with the given curve (lines_per_bscan floats; NULL =
 * the reference's curve), cuda_kernels.cu:408-438 semantics. */
OPE_B200_API int ope_b200_op_sinusoidal_correction(const float* input, const float* curve, int32_t line_width,
                                                   int32_t lines_per_bscan, int32_t num_bscans, float* out);
/* postProcessTruncate: log or linear scaling of lines of line_width interleaved
 * complex values to line_width/2 outputs each (cpu_kernels.tpp:301-378, auto
 * range per line when min == max in log mode). */
OPE_B200_API int ope_b200_op_truncate(const float* input, int32_t log_scaling, float grayscale_max,
                                      float grayscale_min, float addend, float multiplicator, int32_t line_width,
                                      int64_t num_lines, float* out);
/* postProcessBackgroundSubtraction: in[i] - (weight * bg[i % line_width] + offset). */
OPE_B200_API int ope_b200_op_background_subtraction(const float* input, const float* background_line, float weight,
                                                    float offset, int32_t line_width, int64_t samples, float* out);

/* Test hook, no reference counterpart: the next launch of this context skips
 * its first input copy, so its bounded wait runs out after `timeout_us`; the
 * kernel then records a status that ope_b200_synchronize / process_host
 * report, and the context stays usable. */
OPE_B200_API int ope_b200_test_inject_copy_stall(ope_b200_ctx* ctx, uint32_t timeout_us);
/* Test hook, no reference counterpart: the next launch of this context issues
 * its first input copies as usual but treats each CTA's first wait as run out,
 * so every CTA takes the timeout path with its copy still in flight or just
 * landed: it waits that copy out (a second bound) before returning and records
 * the timeout status alone; the context stays usable. */
OPE_B200_API int ope_b200_test_inject_wait_abort(ope_b200_ctx* ctx);

/* ABI version and build information. */
OPE_B200_API int ope_b200_abi_version(void);
/* 1 if the library can run on device `device` (an sm_100 GPU is present). */
OPE_B200_API int ope_b200_device_supported(int32_t device);

#ifdef __cplusplus
}
#endif

#endif /* OPE_B200_H */
