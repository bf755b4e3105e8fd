/*
 * fcwt_b200.h — C ABI of the B200-native fCWT transform path.
 *
 * Plain C types only: pointers, sizes and status codes. Every entry point
 * returns FCWT_OK (0) or an FCWT_ERR_* code; fcwt_last_error() returns a
 * message for the calling thread's last failure.
 *
 * Signal and output pointers may be host or device memory (detected per call).
 * With host pointers the call copies in and out and returns when the output is
 * written. With device pointers the call only enqueues work on the context's
 * stream; fcwt_synchronize() waits for it and reports device-side errors.
 *
 * Each entry point names the reference interface it replaces
 * (reference = fastlib/fCWT, paths inside that project).
 */
#ifndef FCWT_B200_H
#define FCWT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes */
#define FCWT_OK 0
#define FCWT_ERR_INVALID 1     /* bad argument (size, pointer, scale, flag)            */
#define FCWT_ERR_CUDA 2        /* CUDA runtime error                                   */
#define FCWT_ERR_NOMEM 3       /* device or host allocation failed                     */
#define FCWT_ERR_UNSUPPORTED 4 /* valid request outside what this build implements     */
#define FCWT_ERR_DEVICE 5      /* a kernel reported an error (e.g. a bounded wait expired) */
#define FCWT_ERR_IO 6          /* plan file could not be read or written               */

/* ---- scale distributions: same values as enum SCALETYPE, src/fcwt/fcwt.h:65 */
#define FCWT_LINSCALES 0
#define FCWT_LOGSCALES 1
#define FCWT_LINFREQS 2

/* ---- transform flags */
#define FCWT_NORM (1u << 0)           /* divide by N: FCWT(..., use_normalization=true) */
#define FCWT_SCALAR_TRUNC (1u << 1)   /* truncation rule of the reference's non-AVX build */
#define FCWT_EXACT_SUPPORT (1u << 2)  /* also evaluate bins whose weight is < 2^-36 of the peak */
#define FCWT_CONTINUOUS (1u << 3)     /* differentiable Morlet: norm*exp(-(2 pi fb (s q/N - 1))^2/2) at every
                                         bin, no mother-table rounding, truncation or reused bins */
#define FCWT_STRICT (1u << 4)         /* refuse frequencies above the Nyquist rate fs/2: the reference's
                                         asserts of src/fcwt/fcwt.cpp:148,167,184, compiled out of its release
                                         builds. For a transform: any scale < 2 (centre frequency fs/scale >
                                         fs/2) fails with FCWT_ERR_INVALID */
/* Wavelet kinds of the reference's Wavelet interface (fields imag_frequency and
 * doublesided, src/fcwt/fcwt.h:75), for caller tables (fcwt_plan_create_mother
 * / fcwt_cwt_mother), with the semantics of the reference's shipped (AVX)
 * product, src/fcwt/fcwt.cpp:232-273: */
#define FCWT_IMAG_FREQUENCY (1u << 5) /* every product is i * mother[idx] * Ihat[q] */
#define FCWT_DOUBLESIDED (1u << 6)    /* bins b in [N - proc, N) are also written, with weight
                                         mother[idx(N - 1 - b)] on the mirrored spectrum (complex64 output) */
#define FCWT_COMPAT_ALIGN (1u << 7)   /* reproduce the reference's odd-n row shift (src/fcwt/fcwt.cpp:418-426):
                                         its inverse FFT writes through std::align(16, ...), so with a 16-byte
                                         aligned output a row i < fn - 1 whose start is 8 mod 16 (odd n, odd i)
                                         holds y_i[t - 1] at t >= 1 and, at t = 0, the previous row's sample
                                         n left there, normalised twice. Complex64 output, whole plans
                                         (all rows, no decimation), 16-byte aligned output only */

/* ---- output element types */
#define FCWT_OUT_C64 0   /* interleaved float32 (re, im): std::complex<float>      */
#define FCWT_OUT_BF16 1  /* interleaved bfloat16 (re, im), 4 bytes per coefficient */
#define FCWT_OUT_F16 2   /* interleaved float16 (re, im), 4 bytes per coefficient  */
/* Fused epilogues (no reference counterpart: the reference's callers take
 * np.abs(output) afterwards, boilerplate.py:46): the scalogram written
 * directly, one float32 per coefficient (half the bytes of complex64). */
#define FCWT_OUT_POWER 3 /* |W|^2 = re^2 + im^2, float32                          */
#define FCWT_OUT_DB 4    /* 10 log10(|W|^2), float32 (-inf where |W| = 0)         */

typedef struct fcwt_context fcwt_context;
typedef struct fcwt_plan fcwt_plan;

/* ---- library / context */
int fcwt_version(void);
const char* fcwt_last_error(void);
/* One context per device and caller thread; it owns a stream and workspace.
 * Calls on one context are not reentrant. */
int fcwt_context_create(int device, fcwt_context** ctx);
int fcwt_context_destroy(fcwt_context* ctx);
/* Use an external cudaStream_t (passed as void*); NULL restores the context's
 * own stream. Pass (void*)1 (cudaStreamLegacy) for the legacy default stream. */
int fcwt_context_set_stream(fcwt_context* ctx, void* cuda_stream);
/* Wait for all work of the context and report device-side errors. */
int fcwt_synchronize(fcwt_context* ctx);

/* Row engine selection (no reference counterpart: the reference has one CPU
 * path). FCWT_ENGINE_AUTO and FCWT_ENGINE_TENSOR_CORES run every row whose bin
 * window spans at most 16 blocks of 1024 bins (N >= 16384) on the tcgen05
 * tensor-core engine and the other rows on the CUDA-core engine;
 * FCWT_ENGINE_CUDA_CORES runs every row on the CUDA-core engine. Changing the
 * mode drops the context's cached plans; plans created earlier keep the mode
 * they were built with. */
#define FCWT_ENGINE_AUTO 0
#define FCWT_ENGINE_CUDA_CORES 1
#define FCWT_ENGINE_TENSOR_CORES 2
int fcwt_context_set_engine(fcwt_context* ctx, int mode);

/* Profiling: when enabled, every transform of the context records CUDA events
 * around its row-engine launch (on the context's stream). */
int fcwt_profile_enable(fcwt_context* ctx, int enable);
/* Waits for the recorded launches; returns their summed device time in ms,
 * the number of row-engine launches, and the number of kernels this library
 * launched since the previous read (counters reset on read). */
int fcwt_profile_read(fcwt_context* ctx, double* engine_ms, int* engine_launches, int* kernel_launches);

/* ---- host-side helpers (no GPU needed) */
/* find2power, src/fcwt/fcwt.h:154-165 */
int fcwt_find2power(int n);
/* Scales::Scales(wavelet, st, fs, f0, f1, fn) + getScales, src/fcwt/fcwt.cpp:111-158 */
int fcwt_scales(int scaletype, int fs, float f0, float f1, int fn, float* scales_out);
/* The same with flags: FCWT_STRICT makes f1 > fs/2 (any scale type) and, for
 * LOGSCALES, f0 >= f1 an FCWT_ERR_INVALID (the reference asserts
 * f1 <= fs/2 in each calculate_*_array, src/fcwt/fcwt.cpp:148,167,184). */
int fcwt_scales_checked(int scaletype, int fs, float f0, float f1, int fn, unsigned flags, float* scales_out);
/* Scales::getFrequencies, src/fcwt/fcwt.cpp:133-137 */
int fcwt_frequencies(const float* scales, int fn, int fs, float* freqs_out);
/* Morlet::getSupport, src/fcwt/fcwt.h:88 */
int fcwt_morlet_support(float fb, float scale);
/* Morlet::generate(real, imag, size, scale), src/fcwt/fcwt.cpp:68-84
 * (real/imag must hold 2*fcwt_morlet_support(fb, scale)+1 floats) */
int fcwt_morlet_time(float fb, float scale, int size, float* real, float* imag);
/* Morlet::getWavelet, src/fcwt/fcwt.cpp:86-105 (pn interleaved complex) */
int fcwt_morlet_wavelet(float fb, float scale, float* out_interleaved, int pn);
/* Morlet::generate(int) on the host, src/fcwt/fcwt.cpp:51-67 */
int fcwt_morlet_mother_host(float fb, int N, float* mother_out);
/* Per-row truncation length of daughter_wavelet_multiplication,
 * src/fcwt/fcwt.cpp:197-311 (proc_out: fn ints), and the bin window the
 * device engine evaluates for Morlet(fb) (lo_out/hi_out may be NULL). */
int fcwt_row_truncation(int n, float fb, const float* scales, int fn, int threads, unsigned flags,
                        int* proc_out, int* lo_out, int* hi_out);

/* ---- device: mother table
 * Morlet::generate(int), src/fcwt/fcwt.cpp:51-67, computed by a kernel. */
int fcwt_morlet_mother(fcwt_context* ctx, float fb, int N, float* mother_out);

/* ---- device: transforms
 * FCWT::cwt(float* input, int n, complex<float>* output, Scales*) and the
 * (input, n, scales, output, n1, n2) overload, src/fcwt/fcwt.cpp:532-543,
 * with FCWT(Morlet(fb), threads, optplans, norm) (src/fcwt/fcwt.h:116-120):
 * output row i (of fn) holds the n coefficients of scales[i]. */
int fcwt_cwt(fcwt_context* ctx, const float* input, int n, float fb, const float* scales, int fn,
             int threads, unsigned flags, void* output, int out_type);
/* FCWT::cwt(complex<float>* input, ...), src/fcwt/fcwt.cpp:536-547 (`ccwt`);
 * input is n interleaved complex values. */
int fcwt_ccwt(fcwt_context* ctx, const float* input, int n, float fb, const float* scales, int fn,
              int threads, unsigned flags, void* output, int out_type);

/* Reusable plan (the FFTW-plan analogue): everything that depends only on the
 * shape, scales and flags is computed once. Rows [row_begin, row_end) of the
 * fn scales are produced (row sharding); the stale-bin semantics still follow
 * all fn rows. */
int fcwt_plan_create(fcwt_context* ctx, int n, int is_complex, float fb, const float* scales, int fn,
                     int threads, unsigned flags, int row_begin, int row_end, fcwt_plan** plan);
int fcwt_plan_execute(fcwt_plan* plan, const void* input, void* output, int out_type);
/* Fused decimation epilogues (no reference counterpart: a caller of the
 * reference decimates the [fn][n] output afterwards). Like fcwt_plan_create,
 * but the plan produces rows row_begin, row_begin + row_stride, ... < row_end
 * and in each row the samples t = 0, time_stride, 2 time_stride, ... < n:
 * output [ceil((row_end - row_begin) / row_stride)][ceil(n / time_stride)].
 * time_stride is a power of two; for padded lengths N > 8192 it must be at
 * most N / 8192 (the four-step transform then skips the columns that are not
 * kept, so decimation by D also divides the inverse-transform work by D).
 * Every computed sample equals the undecimated transform's sample; the
 * reused-bin semantics still follow all fn rows. */
int fcwt_plan_create_strided(fcwt_context* ctx, int n, int is_complex, float fb, const float* scales, int fn,
                             int threads, unsigned flags, int row_begin, int row_end, int row_stride,
                             int time_stride, fcwt_plan** plan);
/* Output shape (rows, samples per row) of a single-signal plan. */
int fcwt_plan_output_shape(const fcwt_plan* plan, int* rows, int* cols);
int fcwt_plan_destroy(fcwt_plan* plan);
/* A caller-supplied wavelet: the reference's FCWT::cwt takes any Wavelet*
 * and uses the table its generate(N) fills (src/fcwt/fcwt.cpp:504-505,
 * fcwt.h:67-79). `mother` (host memory) holds that table, N =
 * 2^find2power(n) floats. Truncation,
 * indices and reused bins follow the reference exactly as for Morlet.
 * FCWT_IMAG_FREQUENCY / FCWT_DOUBLESIDED in `flags` select the other wavelet
 * kinds of the reference's product (a doublesided row is computed as two
 * single-sided passes, the second on the spectrum shifted by one bin, and a
 * combine; complex64 output only). */
int fcwt_plan_create_mother(fcwt_context* ctx, int n, int is_complex, const float* mother, int mother_size,
                            const float* scales, int fn, int threads, unsigned flags, int row_begin, int row_end,
                            fcwt_plan** plan);
int fcwt_cwt_mother(fcwt_context* ctx, const void* input, int n, int is_complex, const float* mother,
                    int mother_size, const float* scales, int fn, int threads, unsigned flags, void* output,
                    int out_type);
/* Introspection (no reference counterpart): rows the plan produces and how many
 * of them the tensor-core engine runs (the rest run on the CUDA-core engine). */
int fcwt_plan_stats(const fcwt_plan* plan, int* rows, int* tensor_core_rows);

/* Batched plan: nsig signals (lengths ns[s], scale grids scales[s] of fns[s]
 * rows, one Morlet(fb)) transformed by one forward-FFT sequence per padded
 * length and ONE persistent row-engine launch that interleaves the work of
 * all signals. No reference counterpart (the reference loops FCWT::cwt per
 * channel); each signal's rows equal FCWT::cwt of that signal. nsig <= 1024. */
int fcwt_plan_create_batched(fcwt_context* ctx, int nsig, const int* ns, int is_complex, float fb,
                             const float* const* scales, const int* fns, int threads, unsigned flags,
                             fcwt_plan** plan);
/* inputs[s] / outputs[s]: per-signal buffers (host or device; output of
 * signal s is fns[s] x ns[s] values). */
int fcwt_plan_execute_batched(fcwt_plan* plan, const void* const* inputs, void* const* outputs, int out_type);
/* Same, for device buffers only, replayed from a CUDA graph: the first call
 * (and any call with different pointers or output type) captures the whole
 * sequence on the context's stream; later calls launch the graph. */
int fcwt_plan_execute_graph(fcwt_plan* plan, const void* const* inputs, void* const* outputs, int out_type);

/* ---- differentiable Morlet CWT (FCWT_CONTINUOUS forward)
 * No reference counterpart (the reference has no gradients). Backward of
 * y[b,i,t] = c * IFFT_N(FFT_N(x_b) * g_i)[t], g_i(q) = norm*exp(-u^2/2),
 * u = 2 pi fb (fs/freqs[i] * q/N - 1), c = 1/N with FCWT_NORM, for a batch of
 * `batch` real signals of n samples and fn rows. Given grad_out = dL/dy*
 * (complex64 [batch][fn][n], torch convention: dL = Re<grad_out, dy>) it writes
 * grad_x (float32 [batch][n]) and returns dL/dfb and dL/dfreqs[i] in host
 * doubles. x, grad_out, grad_x: device pointers; freqs: host array. The input
 * spectra are recomputed, not stored. */
int fcwt_morlet_cwt_backward(fcwt_context* ctx, const float* x, int n, int batch, float fb, const float* freqs,
                             int fn, float fs, unsigned flags, const void* grad_out, float* grad_x, double* grad_fb,
                             double* grad_freqs);

/* ---- tuning files
 * FCWT::create_FFT_optimization_plan(maxsize, flags), src/fcwt/fcwt.cpp:313-374:
 * for N = 2^11 .. 2^ceil(log2 maxsize), times the engine's scheduling
 * choices and writes "n<N>_t<threads>.wis" into `directory` (NULL: current
 * directory). level 0..3 mirrors FFTW_ESTIMATE/MEASURE/PATIENT/EXHAUSTIVE. */
int fcwt_create_optimization_plan(fcwt_context* ctx, int maxsize, int threads, int level,
                                  const char* directory);
/* FCWT::load_FFT_optimization_plan, src/fcwt/fcwt.cpp:376-393: use the
 * choices stored for (N, threads) by later transforms of this context.
 * Returns FCWT_ERR_IO when the file is missing or malformed (the context then
 * keeps its defaults). */
int fcwt_load_optimization_plan(fcwt_context* ctx, int n, int threads, const char* directory);

/* ---- allocation-free transform
 * No counterpart in the reference. Same result as fcwt_cwt (real input,
 * complex64 output) for callers that cannot allocate device memory: code on a
 * real-time thread (audio/sensor callbacks) where cudaMalloc may block and
 * synchronize the device, plug-ins whose host framework owns all device
 * memory, and callers that fix their footprint at start-up. The call
 * allocates nothing: all its device workspace is one static array of about
 * 2.3 MB inside the library (held on every GPU that loads the library).
 * Limits: n <= 16384, fn <= 1024, at most 8 stale-bin tables; larger
 * requests fail with FCWT_ERR_INVALID. input/output must be device pointers of
 * the current device; scales is a host array (other pointers fail with
 * FCWT_ERR_INVALID); work is enqueued on `stream` (a cudaStream_t, NULL =
 * legacy default stream). The call makes no host-to-device copies: its
 * descriptors reach the device as kernel parameters, so it does not wait for
 * earlier work in the stream (host-side planning still uses the C++ heap).
 * The first call on a device resolves the array's address
 * (cudaGetSymbolAddress) and configures the kernels for that device
 * (cudaFuncSetAttribute). That address is kept for the life of the process:
 * do not call cudaDeviceReset while the library is in use. All calls share the array: calls whose GPU work overlaps
 * race; serialize them on one stream. With status != NULL the call waits for
 * its work and stores the device error word there (0 = ok); with status ==
 * NULL it neither waits nor reads that word, so a device-side error is not
 * reported by this call. */
int fcwt_cwt_noalloc(const float* input, int n, float fb, const float* scales, int fn, int threads,
                     unsigned flags, void* output, void* stream, int* status);

#ifdef __cplusplus
}
#endif

#endif /* FCWT_B200_H */
