// spectral.cu -- STFT, Welch power spectral density and magnitude-squared
// coherence as batched single launches.
//
// Reference: STFT.analyze (Sources/MetalFFT/DSP/STFT.swift:79-108),
// PSD.welch (DSP/PSD.swift:18-58) and PSD.coherence (DSP/PSD.swift:71-134)
// loop over frames on the host: per frame a vDSP window multiply, a complex
// pack with zero imaginary part, one GPU forward FFT of fftSize points and a
// CPU accumulation.  Here every frame of the signal is transformed in one
// launch:
//  * two real frames travel as the real and imaginary parts of one complex
//    line (STFT and Welch: frames 2p and 2p+1; coherence: frame f of a and of
//    b); the Hermitian split A_k = (Z_k + conj Z_{n-k})/2,
//    B_k = (Z_k - conj Z_{n-k})/(2i) recovers both spectra, so a pair of
//    frames costs one transform instead of two;
//  * the window multiply is fused into the load (each thread keeps its 16
//    window values in registers across frames);
//  * Welch and coherence sums accumulate per bin in shared memory (global
//    memory when it does not fit, coherence at 16384) owned by one thread per
//    bin, are written per walker and summed over walkers in a fixed order,
//    then normalised: deterministic, no atomics.
#include <vector>

#include "capi_internal.h"
#include "stockham.cuh"

namespace mfft {

namespace {

constexpr int SP_E = 16;

template <int FFT>
struct SpGeom {
    static constexpr int T = FFT / SP_E;
    static constexpr int LINES = T >= 128 ? 1 : 128 / T;  // lines (walkers) per CTA
    static constexpr int THREADS = T * LINES;
    static constexpr bool WS = (T <= 32);
    static constexpr int XCH = LINES * spad_size(FFT);  // exchange area, float2
    // accumulation kernels: up to three CTAs of <= 256 threads per SM (80
    // registers at fft 4096, no spills)
    static constexpr int MINB = THREADS <= 256 ? 3 : 1;
    // per-line accumulator planes: Welch 1 (power), coherence 4 (Sxx, Syy, Re, Im Sxy)
    template <int PLANES>
    static constexpr bool acc_smem() {
        return XCH * 8 + LINES * PLANES * FFT * 4 <= 227 * 1024;
    }
    template <int PLANES>
    static constexpr int smem_bytes() {
        return XCH * 8 + (acc_smem<PLANES>() ? LINES * PLANES * FFT * 4 : 0);
    }
};

// Z (natural order in v, thread t holds k = t + m*T) -> A, B spectra of the
// real and imaginary inputs, handed bin by bin to use(m, A, B) so that no
// second and third spectrum array is kept in registers; Z_{n-k} comes
// through the exchange area.
template <int FFT, bool WS, class Buf, class Use>
__device__ __forceinline__ void hermitian_split(const float2 (&v)[SP_E], int t, const Buf& buf, Use&& use) {
    constexpr int T = FFT / SP_E;
#pragma unroll
    for (int m = 0; m < SP_E; ++m) buf[t + m * T] = v[m];
    line_sync<WS>();
#pragma unroll
    for (int m = 0; m < SP_E; ++m) {
        const int k = t + m * T;
        const float2 zc = cconj(buf[(FFT - k) & (FFT - 1)]);
        const float2 A = make_float2(0.5f * (v[m].x + zc.x), 0.5f * (v[m].y + zc.y));
        const float2 d = make_float2(0.5f * (v[m].x - zc.x), 0.5f * (v[m].y - zc.y));
        use(m, A, make_float2(d.y, -d.x));  // B = d / i
    }
    line_sync<WS>();
}

// frames (2p, 2p+1) of x, windowed, as one complex line
template <int FFT>
__device__ __forceinline__ void load_pair(const float* __restrict__ x, long long frames, int hop, long long p, int t,
                                          const float (&w)[SP_E], float2 (&v)[SP_E]) {
    constexpr int T = FFT / SP_E;
    const long long f0 = 2 * p;
    const bool ok0 = f0 < frames, ok1 = f0 + 1 < frames;
    const float* x0 = x + f0 * hop + t;
#pragma unroll
    for (int m = 0; m < SP_E; ++m) {
        const float re = ok0 ? __ldcs(x0 + m * T) * w[m] : 0.f;
        const float im = ok1 ? __ldcs(x0 + hop + m * T) * w[m] : 0.f;
        v[m] = make_float2(re, im);
    }
}

template <int FFT>
__global__ void __launch_bounds__(SpGeom<FFT>::THREADS)
    k_stft(const float* __restrict__ x, long long frames, int hop, const float* __restrict__ win,
           const float2* __restrict__ tw, float2* __restrict__ spec, float* __restrict__ power) {
    using G = SpGeom<FFT>;
    constexpr int T = G::T;
    extern __shared__ __align__(16) float2 smem[];
    const int lf = threadIdx.x / T, t = threadIdx.x % T;
    const PadLine buf{smem + lf * spad_size(FFT)};
    const long long p = (long long)blockIdx.x * G::LINES + lf;  // frame pair (idle lines still sync)
    float w[SP_E];
#pragma unroll
    for (int m = 0; m < SP_E; ++m) w[m] = __ldg(win + t + m * T);
    float2 v[SP_E];
    load_pair<FFT>(x, frames, hop, p, t, w, v);
    fft_regs<FFT, SP_E, G::WS>(v, t, buf, tw);
    const long long f0 = 2 * p;
    const bool ok0 = f0 < frames, ok1 = f0 + 1 < frames;
    float2* s0 = spec ? spec + f0 * FFT + t : nullptr;
    float* p0 = power ? power + f0 * FFT + t : nullptr;
    hermitian_split<FFT, G::WS>(v, t, buf, [&](int m, float2 A, float2 B) {
        if (s0) {
            if (ok0) __stcs(s0 + m * T, A);
            if (ok1) __stcs(s0 + FFT + m * T, B);
        }
        if (p0) {
            if (ok0) __stcs(p0 + m * T, A.x * A.x + A.y * A.y);
            if (ok1) __stcs(p0 + FFT + m * T, B.x * B.x + B.y * B.y);
        }
    });
}

// Welch (COH = false): walker u owns frame pairs [u*per, (u+1)*per) of x and
// sums |A|^2 + |B|^2 per bin.  Coherence (COH = true): walker u owns frames
// [u*per, (u+1)*per); line = frame f of a (re) and of b (im); sums |A|^2,
// |B|^2, Re and Im of A conj(B).  Sums land in part[u][plane][FFT].
template <int FFT, bool COH>
__global__ void __launch_bounds__(SpGeom<FFT>::THREADS, SpGeom<FFT>::MINB)
    k_spec_acc(const float* __restrict__ a, const float* __restrict__ b, long long frames, int hop,
               const float* __restrict__ win, const float2* __restrict__ tw, long long work, long long per,
               float* __restrict__ part) {
    using G = SpGeom<FFT>;
    constexpr int T = G::T;
    constexpr int PLANES = COH ? 4 : 1;
    constexpr bool ACC_SMEM = G::template acc_smem<PLANES>();
    extern __shared__ __align__(16) float2 smem[];
    const int lf = threadIdx.x / T, t = threadIdx.x % T;
    const PadLine buf{smem + lf * spad_size(FFT)};
    const long long u = (long long)blockIdx.x * G::LINES + lf;
    float* acc = ACC_SMEM ? reinterpret_cast<float*>(smem + G::XCH) + lf * PLANES * FFT : part + u * PLANES * FFT;
#pragma unroll
    for (int pl = 0; pl < PLANES; ++pl)
#pragma unroll
        for (int m = 0; m < SP_E; ++m) acc[pl * FFT + t + m * T] = 0.f;
    float w[SP_E];
#pragma unroll
    for (int m = 0; m < SP_E; ++m) w[m] = __ldg(win + t + m * T);
    const long long i0 = u * per;
    for (long long it = 0; it < per; ++it) {  // same count on every line of the CTA
        const long long i = i0 + it;
        const bool active = i < work;
        float2 v[SP_E];
        if constexpr (COH) {
            const float* pa = a + i * hop + t;
            const float* pb = b + i * hop + t;
#pragma unroll
            for (int m = 0; m < SP_E; ++m)
                v[m] = active ? make_float2(__ldcs(pa + m * T) * w[m], __ldcs(pb + m * T) * w[m]) : make_float2(0.f, 0.f);
        } else {
            load_pair<FFT>(a, active ? frames : 0, hop, i, t, w, v);
        }
        fft_regs<FFT, SP_E, G::WS>(v, t, buf, tw);
        hermitian_split<FFT, G::WS>(v, t, buf, [&](int m, float2 A, float2 B) {
            const int k = t + m * T;
            const float pa = A.x * A.x + A.y * A.y, pb = B.x * B.x + B.y * B.y;
            if constexpr (COH) {
                acc[k] += pa;
                acc[FFT + k] += pb;
                acc[2 * FFT + k] += A.x * B.x + A.y * B.y;
                acc[3 * FFT + k] += A.y * B.x - A.x * B.y;
            } else {
                acc[k] += pa + pb;  // B is zero when frame 2i+1 does not exist
            }
        });
    }
    if constexpr (ACC_SMEM) {
        float* dst = part + u * PLANES * FFT;
#pragma unroll
        for (int pl = 0; pl < PLANES; ++pl)
#pragma unroll
            for (int m = 0; m < SP_E; ++m) dst[pl * FFT + t + m * T] = acc[pl * FFT + t + m * T];
    }
}

// one thread per bin: fixed-order sum over walkers, then the normalisation
template <bool COH>
__global__ void k_spec_finish(const float* __restrict__ part, long long units, int fft, float scale,
                              float* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= fft) return;
    constexpr int PLANES = COH ? 4 : 1;
    double s[PLANES];
#pragma unroll
    for (int pl = 0; pl < PLANES; ++pl) s[pl] = 0.0;
    for (long long u = 0; u < units; ++u)
#pragma unroll
        for (int pl = 0; pl < PLANES; ++pl) s[pl] += part[(u * PLANES + pl) * fft + k];
    if constexpr (COH) {
        const double den = s[0] * s[1];
        out[k] = den > 0.0 ? (float)((s[2] * s[2] + s[3] * s[3]) / den) : 0.f;
    } else {
        out[k] = (float)(s[0] * scale);
    }
}

struct SpKernels {
    int fft, threads, lines;
    int smem_stft, smem_welch, smem_coh;
    cudaError_t (*prepare)();
    void (*stft)(dim3, cudaStream_t, const float*, long long, int, const float*, const float2*, float2*, float*);
    void (*acc)(bool, dim3, cudaStream_t, const float*, const float*, long long, int, const float*, const float2*,
                long long, long long, float*);
    int (*acc_ctas_per_sm)(bool);
};

template <int FFT>
cudaError_t sp_prepare() {
    using G = SpGeom<FFT>;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_stft<FFT>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::XCH * 8))) return e;
    if ((e = cudaFuncSetAttribute(k_spec_acc<FFT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  G::template smem_bytes<1>())))
        return e;
    return cudaFuncSetAttribute(k_spec_acc<FFT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                G::template smem_bytes<4>());
}
template <int FFT>
void sp_stft(dim3 grid, cudaStream_t s, const float* x, long long frames, int hop, const float* w, const float2* tw,
             float2* spec, float* power) {
    k_stft<FFT><<<grid, SpGeom<FFT>::THREADS, SpGeom<FFT>::XCH * 8, s>>>(x, frames, hop, w, tw, spec, power);
}
template <int FFT>
void sp_acc(bool coh, dim3 grid, cudaStream_t s, const float* a, const float* b, long long frames, int hop,
            const float* w, const float2* tw, long long work, long long per, float* part) {
    using G = SpGeom<FFT>;
    if (coh)
        k_spec_acc<FFT, true><<<grid, G::THREADS, G::template smem_bytes<4>(), s>>>(a, b, frames, hop, w, tw, work,
                                                                                    per, part);
    else
        k_spec_acc<FFT, false><<<grid, G::THREADS, G::template smem_bytes<1>(), s>>>(a, b, frames, hop, w, tw, work,
                                                                                     per, part);
}

template <int FFT>
int sp_acc_occ(bool coh) {
    using G = SpGeom<FFT>;
    int occ = 0;
    cudaError_t e = coh ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spec_acc<FFT, true>, G::THREADS,
                                                                        G::template smem_bytes<4>())
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spec_acc<FFT, false>, G::THREADS,
                                                                        G::template smem_bytes<1>());
    return (e == cudaSuccess && occ > 0) ? occ : 1;
}

#define MFFT_SPK(F)                                                                                         \
    {F, SpGeom<F>::THREADS, SpGeom<F>::LINES, SpGeom<F>::XCH * 8, SpGeom<F>::template smem_bytes<1>(),     \
     SpGeom<F>::template smem_bytes<4>(), &sp_prepare<F>, &sp_stft<F>, &sp_acc<F>, &sp_acc_occ<F>}

const SpKernels g_spk[] = {MFFT_SPK(64),   MFFT_SPK(128),  MFFT_SPK(256),  MFFT_SPK(512),  MFFT_SPK(1024),
                           MFFT_SPK(2048), MFFT_SPK(4096), MFFT_SPK(8192), MFFT_SPK(16384)};

const SpKernels* find_spk(int fft) {
    for (const auto& k : g_spk)
        if (k.fft == fft) return &k;
    return nullptr;
}

}  // namespace

}  // namespace mfft

using namespace mfft;

struct mfft_spectral {
    mfft_ctx* ctx = nullptr;
    int64_t fft = 0, hop = 0;
    const SpKernels* k = nullptr;
    float2* tw = nullptr;
    float* window = nullptr;  // device
    double window_sumsq = 0;
    float* part = nullptr;    // walker sums
    long long part_floats = 0;
    int occ_welch = 0, occ_coh = 0;  // resident CTAs per SM of the accumulation kernels
};

extern "C" int mfft_spectral_destroy(mfft_spectral* s) {
    if (!s) return MFFT_SUCCESS;
    DeviceGuard g(s->ctx->device);
    cudaFree(s->window);
    cudaFree(s->part);
    delete s;
    return MFFT_SUCCESS;
}

extern "C" int mfft_spectral_create(mfft_ctx* ctx, int64_t fft_size, int64_t hop_size, int window_kind,
                                    double kaiser_beta, mfft_spectral** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    *out = nullptr;
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    if (!is_pow2_in(fft_size, 64, MFFT_MAX_SINGLE_N))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, fft_size, -1, -1,
                         "Unsupported FFT size: %lld. Supported: powers of two 64..16384", (long long)fft_size);
    if (hop_size < 1 || hop_size > (1LL << 30))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, hop_size, -1, "hop size must be in [1, 2^30], got %lld",
                         (long long)hop_size);
    std::vector<float> w((size_t)fft_size);
    int st = mfft_window(window_kind, fft_size, kaiser_beta, w.data());
    if (st) return st;
    DeviceGuard g(ctx->device);
    mfft_spectral* s = new mfft_spectral();
    s->ctx = ctx;
    s->fft = fft_size;
    s->hop = hop_size;
    s->k = find_spk((int)fft_size);
    for (float v : w) s->window_sumsq += (double)v * (double)v;
    st = line_twiddles(ctx, (int)fft_size, &s->tw);
    cudaError_t e = cudaSuccess;
    if (!st) e = s->k->prepare();
    if (!st && e != cudaSuccess) st = cuda_error(e, "spectral kernel attributes");
    if (!st) {
        e = cudaMalloc(&s->window, sizeof(float) * fft_size);
        if (e == cudaSuccess) e = cudaMemcpy(s->window, w.data(), sizeof(float) * fft_size, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "window: %s", cudaGetErrorString(e));
    }
    if (st) {
        mfft_spectral_destroy(s);
        return st;
    }
    *out = s;
    return MFFT_SUCCESS;
}

extern "C" int64_t mfft_stft_frame_count(const mfft_spectral* s, int64_t sample_count) {
    if (!s || sample_count < s->fft) return 0;
    return (sample_count - s->fft) / s->hop + 1;
}

namespace {

// Host-array call with several inputs and outputs: stage, run, copy back, wait.
struct HostBuf {
    const void* host_in;
    void* host_out;
    size_t bytes;
    void* dev;
};
int host_call(mfft_ctx* ctx, std::vector<HostBuf>& bufs, const std::function<int(cudaStream_t)>& body) {
    cudaStream_t s = ctx->stream;
    int st = MFFT_SUCCESS;
    cudaError_t e = cudaSuccess;
    for (auto& b : bufs) {
        b.dev = nullptr;
        if (!b.bytes) continue;
        e = cudaMallocAsync(&b.dev, b.bytes, s);
        if (e != cudaSuccess) {
            st = set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "Device buffer allocation failed: %s", cudaGetErrorString(e));
            break;
        }
        if (b.host_in) {
            e = cudaMemcpyAsync(b.dev, b.host_in, b.bytes, cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) {
                st = cuda_error(e, "host to device copy");
                break;
            }
        }
    }
    if (!st) st = body(s);
    if (!st)
        for (auto& b : bufs)
            if (b.host_out && b.dev) {
                e = cudaMemcpyAsync(b.host_out, b.dev, b.bytes, cudaMemcpyDeviceToHost, s);
                if (e != cudaSuccess) {
                    st = cuda_error(e, "device to host copy");
                    break;
                }
            }
    for (auto& b : bufs)
        if (b.dev) cudaFreeAsync(b.dev, s);
    e = cudaStreamSynchronize(s);
    if (!st && e != cudaSuccess) st = cuda_error(e, "execution");
    if (!st) st = check_device_error(ctx);
    return st;
}

int check_flags(int flags) {
    if (flags != MFFT_HOST_MEMORY && flags != MFFT_DEVICE_MEMORY)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown flags %d", flags);
    return MFFT_SUCCESS;
}

int stft_device(mfft_spectral* s, const float* x, long long frames, float2* spec, float* power, cudaStream_t st) {
    const long long pairs = (frames + 1) / 2;
    const long long ctas = (pairs + s->k->lines - 1) / s->k->lines;
    if (ctas <= 0) return MFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, frames, -1, "too many frames");
    s->k->stft(dim3((unsigned)ctas), st, x, frames, (int)s->hop, s->window, s->tw, spec, power);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "STFT launch");
    return MFFT_SUCCESS;
}

// walkers over `work` items (pairs or frames): one CTA per resident slot
int acc_device(mfft_spectral* s, bool coh, const float* a, const float* b, long long frames, long long work,
               float scale, float* out, cudaStream_t st) {
    const int lines = s->k->lines;
    int& occ = coh ? s->occ_coh : s->occ_welch;
    if (!occ) occ = s->k->acc_ctas_per_sm(coh);
    long long units = (long long)s->ctx->sms * occ * lines;
    if (units > work) units = work;
    if (units < 1) units = 1;
    const long long per = work > 0 ? (work + units - 1) / units : 0;
    units = per > 0 ? (work + per - 1) / per : 1;
    const long long ctas = (units + lines - 1) / lines;
    const long long slots = ctas * lines;
    const int planes = coh ? 4 : 1;
    const long long need = slots * planes * s->fft;
    if (need > s->part_floats) {
        cudaFree(s->part);
        s->part = nullptr;
        s->part_floats = 0;
        cudaError_t e = cudaMalloc(&s->part, sizeof(float) * need);
        if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "spectral sums: %s", cudaGetErrorString(e));
        s->part_floats = need;
    }
    s->k->acc(coh, dim3((unsigned)ctas), st, a, b, frames, (int)s->hop, s->window, s->tw, work, per, s->part);
    if (coh) k_spec_finish<true><<<(unsigned)((s->fft + 255) / 256), 256, 0, st>>>(s->part, slots, (int)s->fft, scale, out);
    else k_spec_finish<false><<<(unsigned)((s->fft + 255) / 256), 256, 0, st>>>(s->part, slots, (int)s->fft, scale, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "spectral launch");
    return MFFT_SUCCESS;
}

}  // namespace

extern "C" int mfft_stft_analyze(mfft_spectral* s, const float* signal, int64_t n, void* spectra, float* power,
                                 int flags, void* stream) {
    if (!s) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "spectral handle is NULL");
    int st = check_flags(flags);
    if (st) return st;
    if (n < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, n, -1, "signal length must be >= 0");
    const long long frames = mfft_stft_frame_count(s, n);
    if (frames > 0 && !signal) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL signal");
    if (frames == 0) return MFFT_SUCCESS;
    DeviceGuard g(s->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY)
        return stft_device(s, signal, frames, (float2*)spectra, power, (cudaStream_t)stream);
    const size_t nb = (size_t)frames * s->fft;
    std::vector<HostBuf> bufs = {{signal, nullptr, (size_t)n * 4, nullptr},
                                 {nullptr, spectra, spectra ? nb * 8 : 0, nullptr},
                                 {nullptr, power, power ? nb * 4 : 0, nullptr}};
    return host_call(s->ctx, bufs, [&](cudaStream_t cs) {
        return stft_device(s, (const float*)bufs[0].dev, frames, (float2*)bufs[1].dev, (float*)bufs[2].dev, cs);
    });
}

extern "C" int mfft_psd_welch(mfft_spectral* s, const float* signal, int64_t n, double sample_rate, float* psd,
                              int flags, void* stream) {
    if (!s) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "spectral handle is NULL");
    int st = check_flags(flags);
    if (st) return st;
    if (n < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, n, -1, "signal length must be >= 0");
    if (!psd) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL output");
    const long long frames = mfft_stft_frame_count(s, n);
    if (frames > 0 && !signal) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL signal");
    // PSD.swift:53-56: 1 / (frames * sum(w^2) * sampleRate); no frames: zeros
    const float scale = frames > 0 ? (float)(1.0 / ((double)frames * s->window_sumsq * sample_rate)) : 0.f;
    DeviceGuard g(s->ctx->device);
    const long long pairs = (frames + 1) / 2;
    if (flags == MFFT_DEVICE_MEMORY) {
        if (frames == 0) {
            cudaError_t e = cudaMemsetAsync(psd, 0, sizeof(float) * s->fft, (cudaStream_t)stream);
            return e == cudaSuccess ? MFFT_SUCCESS : cuda_error(e, "PSD zero fill");
        }
        return acc_device(s, false, signal, nullptr, frames, pairs, scale, psd, (cudaStream_t)stream);
    }
    std::vector<HostBuf> bufs = {{signal, nullptr, frames > 0 ? (size_t)n * 4 : 0, nullptr},
                                 {nullptr, psd, (size_t)s->fft * 4, nullptr}};
    return host_call(s->ctx, bufs, [&](cudaStream_t cs) {
        if (frames == 0) {
            cudaError_t e = cudaMemsetAsync(bufs[1].dev, 0, sizeof(float) * s->fft, cs);
            return e == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(e, "PSD zero fill");
        }
        return acc_device(s, false, (const float*)bufs[0].dev, nullptr, frames, pairs, scale, (float*)bufs[1].dev, cs);
    });
}

extern "C" int mfft_psd_coherence(mfft_spectral* s, const float* a, int64_t na, const float* b, int64_t nb,
                                  float* coherence, int flags, void* stream) {
    if (!s) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "spectral handle is NULL");
    int st = check_flags(flags);
    if (st) return st;
    if (na < 0 || nb < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "signal lengths must be >= 0");
    if (!coherence) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL output");
    const long long n = na < nb ? na : nb;  // PSD.swift:98
    const long long frames = mfft_stft_frame_count(s, n);
    if (frames > 0 && (!a || !b)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL signal");
    DeviceGuard g(s->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY) {
        if (frames == 0) {
            cudaError_t e = cudaMemsetAsync(coherence, 0, sizeof(float) * s->fft, (cudaStream_t)stream);
            return e == cudaSuccess ? MFFT_SUCCESS : cuda_error(e, "coherence zero fill");
        }
        return acc_device(s, true, a, b, frames, frames, 1.f, coherence, (cudaStream_t)stream);
    }
    const size_t in_b = frames > 0 ? (size_t)n * 4 : 0;
    std::vector<HostBuf> bufs = {{a, nullptr, in_b, nullptr},
                                 {b, nullptr, in_b, nullptr},
                                 {nullptr, coherence, (size_t)s->fft * 4, nullptr}};
    return host_call(s->ctx, bufs, [&](cudaStream_t cs) {
        if (frames == 0) {
            cudaError_t e = cudaMemsetAsync(bufs[2].dev, 0, sizeof(float) * s->fft, cs);
            return e == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(e, "coherence zero fill");
        }
        return acc_device(s, true, (const float*)bufs[0].dev, (const float*)bufs[1].dev, frames, frames, 1.f,
                          (float*)bufs[2].dev, cs);
    });
}
