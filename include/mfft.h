/*
 * mfft.h -- C ABI of libmfft.so, the B200 (sm_100a) implementation of
 * MetalFFT's batched complex FFT path and its direct callers.
 *
 * The reference's public boundary is a Swift API (docs/MetalFFT.swiftinterface
 * :12-266).  Every entry point below names the Swift declaration it replaces;
 * a Swift/C++/Python wrapper re-creates that API on top (the Python mirror is
 * metalfft_b200/__init__.py, the C++ mirror is metalfft_b200/MetalFFT.hpp).
 *
 * Conventions
 *  - Complex data is interleaved complex64: {float re, float im} per element
 *    (the reference's SIMD2<Float>), transform b of a batch at offset b*n.
 *  - Forward is unscaled with the e^{-2*pi*i*j*k/n} kernel
 *    (Sources/MetalFFT/Resources/fft_multisize.metal:70); inverse is
 *    (1/n) * conj(FFT(conj(X))) (Sources/MetalFFT/FFT/MetalFFT.swift:56-65).
 *  - Every function returns an mfft_status; nothing aborts and nothing traps
 *    on the device.  The text of the last error on the calling thread is
 *    returned by mfft_last_error().
 *  - flags: MFFT_HOST_MEMORY (default) means the pointers are host memory;
 *    the call copies in, runs and copies out before returning, which is the
 *    Swift arrays' semantics (MetalFFT.swift:74-84, synchronous like
 *    commitAndWait, Internal/Dispatch.swift:3-10).  MFFT_DEVICE_MEMORY means
 *    the pointers are device memory and the work is only enqueued on
 *    `stream` (a cudaStream_t; NULL = the legacy default stream).  Complex
 *    device buffers of the FFT calls (mfft_exec_c2c, mfft_exec_c2c_tc,
 *    mfft_multi_exec) must be 16-byte aligned, as cudaMalloc and PyTorch
 *    allocations are; others are MFFT_ERR_INVALID_ARGUMENT.
 *  - Handles are single-writer: one thread at a time per handle
 *    (MetalFFT.swift:9).  Context creation is thread-safe.
 */
#ifndef MFFT_H
#define MFFT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MFFT_API __attribute__((visibility("default")))
#else
#define MFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1..9 map one-to-one onto the cases of FFTError
 * (Sources/MetalFFT/Internal/MetalContext.swift:6-30). */
typedef enum mfft_status {
    MFFT_SUCCESS = 0,
    MFFT_ERR_NO_DEVICE = 1,          /* FFTError.noMetalDevice            */
    MFFT_ERR_NO_STREAM = 2,          /* FFTError.noCommandQueue           */
    MFFT_ERR_LIBRARY_BUILD = 3,      /* FFTError.libraryBuildFailed       */
    MFFT_ERR_KERNEL_NOT_FOUND = 4,   /* FFTError.kernelNotFound           */
    MFFT_ERR_EXEC_FAILED = 5,        /* FFTError.commandBufferFailed      */
    MFFT_ERR_INVALID_INPUT_SIZE = 6, /* FFTError.invalidInputSize         */
    MFFT_ERR_BATCH_INPUT_SIZE = 7,   /* FFTError.batchInputSize           */
    MFFT_ERR_UNSUPPORTED_SIZE = 8,   /* FFTError.unsupportedFFTSize       */
    MFFT_ERR_ALLOCATION = 9,         /* FFTError.bufferAllocationFailed   */
    MFFT_ERR_INVALID_ARGUMENT = 10,  /* Swift precondition() traps        */
    MFFT_ERR_TIMEOUT = 11            /* a bounded device-side wait expired */
} mfft_status;

enum {
    MFFT_HOST_MEMORY = 0,
    MFFT_DEVICE_MEMORY = 1
};

enum {
    MFFT_FORWARD = -1,
    MFFT_INVERSE = +1
};

/* Tensor-core variants for mfft_exec_c2c_tc. */
enum {
    MFFT_TC_FP16_SPLIT3 = 1, /* hi/lo FP16 split, 3 products, FP32 accumulate */
    MFFT_TC_BF16 = 2         /* plain BF16 operands, FP32 accumulate          */
};

/* FusedConvolver.Precision (Sources/MetalFFT/DSP/FusedConvolver.swift:27-36)
 * for mfft_conv_set_precision. */
enum {
    MFFT_CONV_FLOAT32 = 0,      /* .float32 (default)                          */
    MFFT_CONV_FP16_PURE = 1,    /* .float16Pure: all butterfly arithmetic FP16 */
    MFFT_CONV_FP16_STORAGE = 2, /* .float16Storage: FP16 storage, FP32 math    */
    MFFT_CONV_FP16_MIXED = 3    /* .float16Mixed: FP16 multiplies, FP32 adds   */
};

/* Window kinds (Sources/MetalFFT/DSP/Window.swift:6-24, WindowType). */
enum {
    MFFT_WINDOW_HANN = 0,
    MFFT_WINDOW_HAMMING = 1,
    MFFT_WINDOW_BLACKMAN = 2,
    MFFT_WINDOW_FLAT_TOP = 3,
    MFFT_WINDOW_KAISER = 4,
    MFFT_WINDOW_RECTANGULAR = 5
};

typedef struct mfft_ctx mfft_ctx;
typedef struct mfft_plan mfft_plan;
typedef struct mfft_conv mfft_conv;
typedef struct mfft_corr mfft_corr;
typedef struct mfft_analyzer mfft_analyzer;
typedef struct mfft_multi mfft_multi;
typedef struct mfft_spectral mfft_spectral;

/* ---- errors ------------------------------------------------------------ */

/* Static text for a status code (FFTError.description, MetalContext.swift:19-29). */
MFFT_API const char* mfft_status_string(int status);

/* Copies the calling thread's last error text (with expected/got/index where
 * the FFTError case carries them) into buf; returns that status. */
MFFT_API int mfft_last_error(char* buf, size_t len);

/* The integer payload of the calling thread's last error:
 * invalidInputSize(expected, got) / batchInputSize(expected, got, batchIndex) /
 * unsupportedFFTSize(n) -> expected = n.  Unused fields are -1. */
MFFT_API int mfft_last_error_detail(int64_t* expected, int64_t* got, int64_t* index);

/* ---- context (MetalContext.shared(), MetalContext.swift:74-142) --------- */

/* The process-wide context for the current CUDA device: created on first use
 * under a lock, then shared.  Never destroy the shared context. */
MFFT_API int mfft_context_shared(mfft_ctx** out);
/* A private context on `device` (-1 = current device). */
MFFT_API int mfft_context_create(int device, mfft_ctx** out);
MFFT_API int mfft_context_destroy(mfft_ctx* ctx);
/* Number of SMs of the context's device (grid sizing). */
MFFT_API int mfft_context_sm_count(const mfft_ctx* ctx);
/* Waits for the device and reports MFFT_ERR_TIMEOUT if any kernel of this
 * context gave up a bounded device-side wait since the last check (host-array
 * calls check after every call; device-pointer calls are checked here). */
MFFT_API int mfft_context_check(mfft_ctx* ctx);

/* Self-test of the failure path (no reference counterpart): runs a kernel
 * whose mbarrier wait can never complete.  The wait gives up after limit_ns
 * (1e3 .. 1e9), records a timeout in the context's device error word and the
 * kernel returns; the call reads and clears that word and returns
 * MFFT_ERR_TIMEOUT.  The context stays usable afterwards. */
MFFT_API int mfft_selftest_bounded_wait(mfft_ctx* ctx, int64_t limit_ns);

/* ---- plans: MetalFFT.init(size:) (MetalFFT.swift:27-51) ---------------- */

/* n: power of two in [64, 2^20].  The reference accepts 64..16384
 * (FFTDescriptor, MetalContext.swift:47-69) and throws unsupportedFFTSize
 * otherwise; sizes above 16384 use the four-step path. */
MFFT_API int mfft_plan_create(mfft_ctx* ctx, int64_t n, mfft_plan** out);
MFFT_API int mfft_plan_destroy(mfft_plan* plan);
MFFT_API int64_t mfft_plan_size(const mfft_plan* plan);
/* Smallest supported size for a kernel of kernel_count taps in the reference's
 * size list, or 0 (Convolver.recommendedFFTSize, Convolve.swift:83-86). */
MFFT_API int64_t mfft_recommended_fft_size(int64_t kernel_count);

/* Batched-kernel variants.  A variant of size n is (radix, lines_per_cta,
 * stages): main radix 8 or 16, lines transformed per CTA, and stages = 0 for
 * the direct-load kernel or the number of line groups a persistent CTA keeps
 * in flight with TMA bulk copies.
 *
 * Autotuner (no reference counterpart; the reference hard-codes one kernel
 * per size, MetalContext.swift:47-69): times every registered variant for
 * size n (64..16384) over `lines` lines (<= 0: 256 MiB worth) and keeps the
 * fastest for this context; appends "n radix lines_per_cta stages" to the file
 * named by $MFFT_TUNE_CACHE, which later contexts read.  Reports the choice. */
MFFT_API int mfft_autotune(mfft_ctx* ctx, int64_t n, int64_t lines, int* radix, int* lines_per_cta,
                           int* stages);
/* Pins a plan (n <= 16384) to one registered variant.
 * MFFT_ERR_KERNEL_NOT_FOUND if that variant is not built. */
MFFT_API int mfft_plan_set_kernel(mfft_plan* plan, int radix, int lines_per_cta, int stages);
/* Lists the registered variants for size n: fills up to cap entries and
 * returns how many exist (host only). */
MFFT_API int mfft_list_kernels(int64_t n, int* radix, int* lines_per_cta, int* stages, int cap);
/* The variant a plan uses and its threads per CTA. */
MFFT_API int mfft_plan_kernel_info(const mfft_plan* plan, int* radix, int* lines_per_cta, int* threads,
                                   int* stages);

/* Four-step split (n > 16384 runs as n1-point column FFTs, a twiddle, and
 * n2 = n/n1-point row FFTs).  The reference fixes one split per size
 * (MetalContext.swift:57-66: 8192 = 64 x 128, 16384 = 128 x 128); here a size
 * takes any n1 with 64 <= n1 <= 1024 and 128 <= n2 <= 1024, and plans start
 * on the split autotuned in the context, else one read from $MFFT_TUNE_CACHE,
 * else n1 = 2^floor(log2(n)/2).
 *
 * mfft_autotune_fourstep times every admissible split over `batch`
 * transforms (<= 0: 512 MiB worth), leaves the plan on the fastest, installs
 * it for later plans of the size in the context, appends "n n1 0 0" to
 * $MFFT_TUNE_CACHE and reports n1.  mfft_plan_set_split pins a plan to n1
 * (MFFT_ERR_INVALID_ARGUMENT if n1 is not admissible); mfft_plan_split reports
 * the plan's split (0, 0 for n <= 16384); mfft_list_splits fills up to cap
 * admissible n1 for size n and returns how many exist (host only). */
MFFT_API int mfft_autotune_fourstep(mfft_plan* plan, int64_t batch, int* n1);
MFFT_API int mfft_plan_set_split(mfft_plan* plan, int64_t n1);
MFFT_API int mfft_plan_split(const mfft_plan* plan, int64_t* n1, int64_t* n2);
MFFT_API int mfft_list_splits(int64_t n, int64_t* n1, int cap);

/* ---- execution --------------------------------------------------------- */

/* Batched C2C.  Replaces forward(_:) (batch = 1, MetalFFT.swift:69-85),
 * forward(input:output:) (MetalFFT.swift:88-104), forward(batch:)
 * (MetalFFT.swift:108-133), inverse(_:) (MetalFFT.swift:56-65) and
 * MultiChannelFFT.forward/inverse (MultiChannelFFT.swift:37-53).
 * direction: MFFT_FORWARD or MFFT_INVERSE (1/n scaled).  batch >= 0
 * (batch == 0 returns at once, as forward(batch: []) returns []).  in == out
 * is allowed. */
MFFT_API int mfft_exec_c2c(mfft_plan* plan, const void* in, void* out, int64_t batch, int direction,
                  int flags, void* stream);

/* Adjoint (backward) of mfft_exec_c2c, for gradients through the FFT (no
 * reference counterpart: the reference has no backward pass; its transform
 * conventions are MetalFFT.swift:56-65 and fft_multisize.metal:70).  For a
 * real loss L of the transform's output y with grad_out = dL/dRe(y) +
 * i dL/dIm(y), writes grad_in = dL/dRe(x) + i dL/dIm(x) for the call's input
 * x, i.e. the conjugate transpose of the transform applied to grad_out:
 *   direction MFFT_FORWARD (y = F x, unscaled):   grad_in = F^H grad_out
 *                                                 = n * inverse(grad_out)
 *   direction MFFT_INVERSE (y = F^H x / n):       grad_in = F grad_out / n
 * Same kernels as mfft_exec_c2c with the direction swapped and the 1/n scale
 * moved to the other side in their stores; same sizes, layout, flags and
 * in-place rule. */
MFFT_API int mfft_exec_c2c_backward(mfft_plan* plan, const void* grad_out, void* grad_in, int64_t batch,
                                    int direction, int flags, void* stream);

/* Tensor-core DFT-as-matmul path (tcgen05 + TMEM) for n = 4096: the B200 form
 * of src/fft_4096_ct_mma.metal:88-206 (simdgroup_float8x8 CT-DIF).  variant:
 * MFFT_TC_FP16_SPLIT3 or MFFT_TC_BF16.  Same layout and scaling as
 * mfft_exec_c2c. */
MFFT_API int mfft_exec_c2c_tc(mfft_plan* plan, const void* in, void* out, int64_t batch,
                     int direction, int variant, int flags, void* stream);

/* Real-input transforms (no reference counterpart: the reference packs real
 * data as complex with a zero imaginary part, Convolve.swift:47-53,
 * FFTAnalyzer.swift:98-100).  n = the plan's size, a power of two 64..16384.
 * r2c: batch lines of n floats -> batch lines of n/2 + 1 complex bins
 * (X_0 .. X_{n/2}; the rest follow from X_{n-k} = conj X_k).  c2r: the
 * inverse, scaled by 1/n.  Two real lines share one complex transform. */
MFFT_API int mfft_exec_r2c(mfft_plan* plan, const float* in, void* out, int64_t batch, int flags, void* stream);
MFFT_API int mfft_exec_c2r(mfft_plan* plan, const void* in, float* out, int64_t batch, int flags, void* stream);

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (an external allocator owns the device, a real-time host reserves
 * memory once at start-up, a plug-in host forbids allocation): the four-step
 * FFT of `batch` lines of length n (powers of two 32768 .. 1048576, else
 * MFFT_ERR_UNSUPPORTED_SIZE) on device pointers, enqueued on `stream`, with
 * no allocation at all.  Its intermediate is a fixed 16 MiB device array (plus
 * ~100 KB of tables) that every GPU loading the library holds until exit;
 * batches go through it in chunks.  The first call on a device does a
 * one-time set-up (launches and waits): make it before any stream capture.
 * Calls share the array, so calls that overlap on the GPU race: serialise
 * them. */
MFFT_API int mfft_fourstep_noalloc(const void* in, void* out, int64_t n, int64_t batch, int direction,
                                   void* stream);

/* ---- mixed sizes in one persistent launch ------------------------------ */

/* One size class: `count` transforms of length n (power of two, 64..2^20)
 * stored back to back starting at complex element `offset` (even) of the
 * in/out buffers.  There is no reference counterpart for a single launch over
 * mixed sizes; it generalises forward(batch:) (MetalFFT.swift:108-133).
 * Sizes up to 4096 run as whole lines, larger ones as four-step transforms
 * (a column pass into an intermediate buffer of the handle holding every
 * four-step point, then a row pass).  One mfft_multi_exec is one kernel
 * launch: persistent CTAs draw 4096-point work items (column items, whole
 * lines, row items) from a device-side descriptor array by atomic ticket, and
 * a row item starts once its transform's column items are counted done (a
 * bounded wait; MFFT_ERR_TIMEOUT when it gives up). */
typedef struct mfft_multi_desc {
    int64_t n;
    int64_t count;
    int64_t offset;
} mfft_multi_desc;

MFFT_API int mfft_multi_create(mfft_ctx* ctx, const mfft_multi_desc* descs, int ndesc,
                      mfft_multi** out);
MFFT_API int mfft_multi_destroy(mfft_multi* m);
/* Total complex elements covered by the descriptors (in and out size). */
MFFT_API int64_t mfft_multi_points(const mfft_multi* m);
MFFT_API int mfft_multi_exec(mfft_multi* m, const void* in, void* out, int direction, int flags,
                    void* stream);

/* ---- Convolver (Convolve.swift:8-87) / FusedConvolver ------------------- */

/* kernel_len < fft_size (the precondition of Convolve.swift:20-21).  The
 * kernel spectrum is computed once on the device (Convolve.swift:27-31). */
MFFT_API int mfft_conv_create(mfft_ctx* ctx, const float* kernel, int64_t kernel_len, int64_t fft_size,
                     mfft_conv** out);
MFFT_API int mfft_conv_destroy(mfft_conv* conv);
MFFT_API int64_t mfft_conv_block_size(const mfft_conv* conv); /* Convolver.blockSize */
MFFT_API int64_t mfft_conv_hop_size(const mfft_conv* conv);   /* Convolver.hopSize   */
MFFT_API int64_t mfft_conv_kernel_len(const mfft_conv* conv);
/* FusedConvolver(kernel:fftSize:precision:) (FusedConvolver.swift:55-83):
 * the arithmetic of later mfft_conv_apply calls, one of MFFT_CONV_*.  The
 * FP16 modes exist for fft_size 4096 only (FusedConvolver.supportedSize,
 * :19); they store X and X*H as half2 and run the FFT exchanges through
 * half2 shared memory, with the inverse's 1/N split as 2^-6 on H and 2^6/N
 * at the end (exact power-of-two scalings that keep every FP16 value 64x
 * below overflow).  mfft_conv_backward stays FP32 in every mode. */
MFFT_API int mfft_conv_set_precision(mfft_conv* conv, int precision);
/* Convolver.apply(to:) / FusedConvolver.apply(to:): out has n + kernel_len - 1
 * samples (Convolve.swift:36-76).  n == 0 gives kernel_len - 1 zeros. */
MFFT_API int mfft_conv_apply(mfft_conv* conv, const float* signal, int64_t n, float* out, int flags,
                    void* stream);
/* Adjoint of apply for a loss L with grad_out = dL/dout (n + kernel_len - 1
 * samples): grad_signal (n samples) and grad_kernel (kernel_len samples).
 * Either output may be NULL.  No reference counterpart (the reference has no
 * backward pass). */
MFFT_API int mfft_conv_backward(mfft_conv* conv, const float* signal, int64_t n, const float* grad_out,
                       float* grad_signal, float* grad_kernel, int flags, void* stream);

/* ---- Correlator (Correlate.swift:7-62) --------------------------------- */

MFFT_API int mfft_corr_create(mfft_ctx* ctx, int64_t fft_size, mfft_corr** out);
MFFT_API int mfft_corr_destroy(mfft_corr* corr);
/* cross(_:_:): out = Re IFFT(FFT(a) * conj(FFT(b))) over fft_size, i.e.
 * out[m] = sum_n a[(n+m) mod fft_size] b[n], inputs zero-padded or truncated
 * to fft_size (Correlate.swift:31-61; the code's lag convention -- its doc
 * comment writes the mirrored sum_n a[n] b[n+m]); fft_size samples written.
 * auto(_:) is cross(a, a). */
MFFT_API int mfft_corr_cross(mfft_corr* corr, const float* a, int64_t na, const float* b, int64_t nb,
                    float* out, int flags, void* stream);

/* ---- FFTAnalyzer (FFTAnalyzer.swift:68-117) ----------------------------- */

/* window coefficients of WindowType.coefficients (Window.swift:12-23). */
MFFT_API int mfft_window(int kind, int64_t n, double kaiser_beta, float* out);
MFFT_API int mfft_analyzer_create(mfft_ctx* ctx, int64_t size, double sample_rate, int window_kind,
                         double kaiser_beta, mfft_analyzer** out);
MFFT_API int mfft_analyzer_destroy(mfft_analyzer* a);
/* analyze(_:offset:): window samples[offset .. offset+size) and FFT them;
 * spectrum receives `size` complex64 bins.  Requires offset + size <= count
 * (the precondition of FFTAnalyzer.swift:108). */
MFFT_API int mfft_analyzer_analyze(mfft_analyzer* a, const float* samples, int64_t count,
                          int64_t offset, void* spectrum, int flags, void* stream);

/* ---- STFT and power spectra (DSP/STFT.swift, DSP/PSD.swift) ------------ */

/* Frames of fft_size samples (power of two 64..16384) every hop_size samples,
 * each multiplied by the window before its FFT: the frame loop of
 * STFT(fftSize:hopSize:window:sampleRate:) (STFT.swift:35-55, 79-107) and of
 * PSD.welch / PSD.coherence (PSD.swift:18-134), run as one launch. */
MFFT_API int mfft_spectral_create(mfft_ctx* ctx, int64_t fft_size, int64_t hop_size, int window_kind,
                                  double kaiser_beta, mfft_spectral** out);
MFFT_API int mfft_spectral_destroy(mfft_spectral* s);
/* STFT.frameCount(for:) (STFT.swift:58-61): (n - fft) / hop + 1, 0 if n < fft. */
MFFT_API int64_t mfft_stft_frame_count(const mfft_spectral* s, int64_t sample_count);
/* STFT.analyze (STFT.swift:79-88): spectra = frames x fft_size complex bins
 * (STFTFrame.complex), power = frames x fft_size |X|^2 (STFTFrame.magnitudes,
 * which are squared magnitudes).  Either output may be NULL. */
MFFT_API int mfft_stft_analyze(mfft_spectral* s, const float* signal, int64_t n, void* spectra, float* power,
                               int flags, void* stream);
/* PSD.welch (PSD.swift:18-58): psd[k] = sum over frames |X_k|^2 /
 * (frames * sum(w^2) * sample_rate), fft_size values; zeros when no frame. */
MFFT_API int mfft_psd_welch(mfft_spectral* s, const float* signal, int64_t n, double sample_rate, float* psd,
                            int flags, void* stream);
/* PSD.coherence (PSD.swift:71-134): over the frames of min(na, nb) samples,
 * C[k] = |sum A conj(B)|^2 / (sum |A|^2 sum |B|^2), 0 where the denominator is
 * not positive; fft_size values. */
MFFT_API int mfft_psd_coherence(mfft_spectral* s, const float* a, int64_t na, const float* b, int64_t nb,
                                float* coherence, int flags, void* stream);

/* PSD.crossSpectral (Sources/MetalFFT/DSP/CrossSpectral.swift:56-152, per-bin
 * kernel Resources/fft_cross_spectral.metal:29-63): `signals` holds `channels`
 * (1..16) real signals of `length` samples each, one after the other.  Frames
 * as in mfft_stft_analyze; per frame and bin p_c = |X_c|^2 and, for the pairs
 * (0,1), (0,2), ..., (0,C-1), (1,2), ..., (C-2,C-1), S_ij = X_i conj(X_j);
 * outputs are means over the frames, fft_size bins each:
 *   power      channels x fft_size      mean p_c
 *   cross      pairs x fft_size complex mean S_ij (NULL allowed for 1 channel)
 *   coherence  pairs x fft_size         coherence_mode 0: mean over frames of
 *              |S_ij|^2 / max(p_i p_j, 1e-30), the reference's formula (1
 *              wherever both channels have power, whatever their relation);
 *              coherence_mode 1: the Welch estimate |mean S_ij|^2 /
 *              (mean p_i mean p_j), 0 where the denominator is not positive.
 * No frames: all outputs zero.  The sample rate only labels bins in the
 * reference and is not an argument.  Device calls keep chunk spectra and
 * partial sums in the handle (grown on demand), so one handle serves one
 * stream at a time. */
MFFT_API int mfft_psd_cross_spectral(mfft_spectral* s, const float* signals, int64_t channels, int64_t length,
                                     float* power, void* cross, float* coherence, int coherence_mode, int flags,
                                     void* stream);

/* ---- SAR range-Doppler chain (src/radar/, src/fft_sar_fused*.metal) ----- */

/* SARParameters (src/radar/sar_simulator.swift:22-67) with the chirp given by
 * its sample count: Tp = chirp_samples / sample_rate, Kr = bandwidth / Tp,
 * lambda = c / carrier, fast time t_r = 2*center_range/c - (range_n/2)/fs +
 * r/fs, slow time eta_p = (p - pulses/2)/prf. */
typedef struct mfft_sar_params {
    int64_t pulses;        /* azimuth lines Na (64 .. 4096, power of two)  */
    int64_t range_n;       /* range samples Nr (512 .. 16384, power of two) */
    int64_t chirp_samples; /* Tp * fs                                       */
    double bandwidth;      /* B, Hz                                         */
    double sample_rate;    /* fs, Hz                                        */
    double prf;            /* Hz                                            */
    double velocity;       /* m/s                                           */
    double carrier;        /* Hz                                            */
    double center_range;   /* m                                             */
} mfft_sar_params;

/* PointTarget (sar_simulator.swift:69-78) plus a reflection phase. */
typedef struct mfft_sar_target {
    double range_m;   /* slant range at closest approach */
    double azimuth_m; /* along-track position            */
    double amplitude;
    double phase;     /* rad */
} mfft_sar_target;

typedef struct mfft_sar mfft_sar;

/* The reference's parameters (SARParameters.init: B = 100 MHz, PRF 1 kHz,
 * v = 100 m/s, X band 10 GHz, 20 km scene centre) with the chirp set by its
 * sample count and time-bandwidth product: fs = chirp_samples * B / tbp. */
MFFT_API int mfft_sar_default_params(int64_t pulses, int64_t range_n, int64_t chirp_samples, double tbp,
                                     mfft_sar_params* out);
/* generateChirpReference (sar_simulator.swift:209-224): the chirp centred
 * circularly at sample 0, range_n complex64 values (host memory). */
MFFT_API int mfft_sar_chirp_reference(const mfft_sar_params* p, void* chirp);
/* SARSimulator.simulate (sar_simulator.swift:93-205) on the device: echoes of
 * the targets (chirp exp(j*pi*Kr*dt^2), two-way phase exp(-j*4*pi*R/lambda),
 * reflection phase) plus complex Gaussian noise at snr_db relative to the mean
 * power of the non-zero samples (addNoise, :161-204) drawn from a
 * counter-based generator of `seed`.  raw: pulses x range_n complex64,
 * device memory, pulse-major. */
MFFT_API int mfft_sar_simulate(mfft_ctx* ctx, const mfft_sar_params* p, const mfft_sar_target* targets,
                               int ntargets, double snr_db, uint64_t seed, void* raw, void* stream);
/* FP16 storage with one power-of-two scale per pulse: raw_h[p][r] * scale[p]
 * ~= raw[p][r].  Device memory. */
MFFT_API int mfft_sar_quantize(mfft_ctx* ctx, int64_t pulses, int64_t range_n, const void* raw,
                               void* raw_h, float* pulse_scale, void* stream);

/* Range matched filter H = conj(FFT(chirp_ref)) (rda_fused_pipeline.swift:
 * 189-196) and the work buffers of one pulses x range_n geometry. */
MFFT_API int mfft_sar_create(mfft_ctx* ctx, const mfft_sar_params* p, const void* chirp_ref, mfft_sar** out);
MFFT_API int mfft_sar_destroy(mfft_sar* sar);
/* Forward image I[k][r] = sum_p W_Na^{pk} u_p[r], u_p = range-compressed pulse
 * p times exp(j*phase[p]): fused range compression (fused_range_compression,
 * src/fft_sar_fused.metal:246-293) then the azimuth FFT with the corner turn
 * folded into its tile loads (azimuthFFT, rda_fused_pipeline.swift:224-242).
 * Input FP16 pulse-major with pulse scales; output FP16 azimuth-major
 * (image[k*range_n + r]) with one scale per range column.  Device memory. */
MFFT_API int mfft_sar_forward(mfft_sar* sar, const void* raw_h, const float* pulse_scale, const float* phase,
                              void* image_h, float* image_scale, void* stream);
/* Precision of the range-compressed intermediate between the range pass and
 * the azimuth pass of later mfft_sar_forward / _backward_phase /
 * _step_graph calls (no reference counterpart; the reference keeps FP32 device
 * data and FP16 only in threadgroup memory, fft_sar_fused_fp16.metal:10-33):
 * MFFT_SAR_RC_FP16 (default): FP16 with one power-of-two scale per pulse,
 * 4 bytes per sample; MFFT_SAR_RC_FP32: FP32, 8 bytes per sample, allocated
 * on first selection (pulses x range_n x 8 bytes).  Input and image stay
 * FP16 in both modes.  The FP32 intermediate is what brings the phase
 * adjoint to within ~1e-5 of the FP64 gradient of the same FP16 input; the
 * FP16 one bounds it near 1e-2. */
enum {
    MFFT_SAR_RC_FP16 = 0,
    MFFT_SAR_RC_FP32 = 1
};
MFFT_API int mfft_sar_set_intermediate(mfft_sar* sar, int precision);
/* Adjoint of L = sum |I|^4 with respect to phase (no reference counterpart):
 * dphi[p] = -sum_r Im(u_p[r] conj(B[p][r])), B = sum_k 4|I|^2 I W^{-pk};
 * the loss goes to *loss (device double).  Recomputes the range pass. */
MFFT_API int mfft_sar_backward_phase(mfft_sar* sar, const void* raw_h, const float* pulse_scale,
                                     const float* phase, float* dphi, double* loss, void* stream);
/* Forward + backward as one CUDA graph, captured on the first call for these
 * pointers and replayed on later calls with the same pointers. */
MFFT_API int mfft_sar_step_graph(mfft_sar* sar, const void* raw_h, const float* pulse_scale, const float* phase,
                                 void* image_h, float* image_scale, float* dphi, double* loss, void* stream);

/* Focused image from the range-Doppler image of mfft_sar_forward (device
 * pointers, same layouts): per Doppler row, range cell migration correction
 * with an 8-tap Hamming-windowed sinc and the azimuth matched filter, then the
 * inverse azimuth FFT (rda_kernels.metal:103-240, rda_fused_pipeline.swift:
 * 248-368).  reference_signs = 1 uses the reference's formulas as written
 * (input read at r - shift, filter exp(-j phase)); 0 uses r + shift and
 * exp(+j phase), which focus the reference's own echo model. */
MFFT_API int mfft_sar_focus(mfft_sar* sar, const void* rd_h, const float* rd_scale, void* focused_h,
                            float* focused_scale, int reference_signs, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MFFT_H */
