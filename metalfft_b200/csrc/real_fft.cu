// real_fft.cu -- real-input forward FFT (n real -> n/2 + 1 complex bins per
// line) and its inverse, n = 64 .. 16384.
//
// The reference has no real-input FFT: its callers pack real samples into
// complex lines with a zero imaginary part (Sources/MetalFFT/DSP/
// Convolve.swift:47-53, Correlate.swift:53-60, FFTAnalyzer.swift:98-100),
// which spends half of every transform on zeros.  Here two real lines travel
// as the real and imaginary parts of one complex line:
//   forward  z = a + i b -> Z = FFT(z); A_k = (Z_k + conj Z_{n-k}) / 2,
//            B_k = (Z_k - conj Z_{n-k}) / (2i), k = 0 .. n/2 (Z_{n-k} through
//            the shared-memory exchange area);
//   inverse  Z_k = A_k + i B_k for all k (the upper half from Hermitian
//            symmetry: A_{n-k} = conj A_k), z = IFFT(Z) / n, a = Re z,
//            b = Im z.
// Inverse outputs are scaled by 1/n like every inverse of this library
// (MetalFFT.swift:56-65).
#include "capi_internal.h"
#include "stockham.cuh"

namespace mfft {

namespace {

constexpr int RF_E = 16;

template <int N>
struct RfGeom {
    static constexpr int T = N / RF_E;
    static constexpr int LINES = T >= 128 ? 1 : 128 / T;  // complex lines (line pairs) per CTA
    static constexpr int THREADS = T * LINES;
    static constexpr bool WS = (T <= 32);
    static constexpr int SMEM = LINES * spad_size(N) * (int)sizeof(float2);
};

template <int N>
__global__ void __launch_bounds__(RfGeom<N>::THREADS) k_r2c(const float* __restrict__ in, float2* __restrict__ out,
                                                             long long batch, const float2* __restrict__ tw) {
    using G = RfGeom<N>;
    constexpr int T = G::T, H = N / 2 + 1;
    extern __shared__ __align__(16) float2 smem[];
    const int lf = threadIdx.x / T, t = threadIdx.x % T;
    const PadLine buf{smem + lf * spad_size(N)};
    const long long pr = (long long)blockIdx.x * G::LINES + lf;  // line pair
    const long long la = 2 * pr;
    const bool ok0 = la < batch, ok1 = la + 1 < batch;
    const float* a = in + la * N + t;
    float2 v[RF_E];
#pragma unroll
    for (int m = 0; m < RF_E; ++m)
        v[m] = make_float2(ok0 ? __ldcs(a + m * T) : 0.f, ok1 ? __ldcs(a + N + m * T) : 0.f);
    fft_regs<N, RF_E, G::WS>(v, t, buf, tw);
#pragma unroll
    for (int m = 0; m < RF_E; ++m) buf[t + m * T] = v[m];
    line_sync<G::WS>();
    float2* oa = out + la * H;
#pragma unroll
    for (int m = 0; m < RF_E; ++m) {
        const int k = t + m * T;
        if (k > N / 2) break;  // bins 0 .. n/2 (k = t + m*T grows with m)
        const float2 zc = cconj(buf[(N - k) & (N - 1)]);
        const float2 A = make_float2(0.5f * (v[m].x + zc.x), 0.5f * (v[m].y + zc.y));
        const float2 d = make_float2(0.5f * (v[m].x - zc.x), 0.5f * (v[m].y - zc.y));
        if (ok0) __stcs(oa + k, A);
        if (ok1) __stcs(oa + H + k, make_float2(d.y, -d.x));
    }
}

template <int N>
__global__ void __launch_bounds__(RfGeom<N>::THREADS) k_c2r(const float2* __restrict__ in, float* __restrict__ out,
                                                             long long batch, const float2* __restrict__ tw) {
    using G = RfGeom<N>;
    constexpr int T = G::T, H = N / 2 + 1;
    extern __shared__ __align__(16) float2 smem[];
    const int lf = threadIdx.x / T, t = threadIdx.x % T;
    const PadLine buf{smem + lf * spad_size(N)};
    const long long pr = (long long)blockIdx.x * G::LINES + lf;
    const long long la = 2 * pr;
    const bool ok0 = la < batch, ok1 = la + 1 < batch;
    const float2* ia = in + la * H;
    float2 v[RF_E];
#pragma unroll
    for (int m = 0; m < RF_E; ++m) {
        // Z_k = A_k + i B_k; for k > n/2, A_k = conj A_{n-k}, B_k = conj B_{n-k}
        const int k = t + m * T;
        const int kk = k <= N / 2 ? k : N - k;
        float2 A = ok0 ? __ldg(ia + kk) : make_float2(0.f, 0.f);
        float2 B = ok1 ? __ldg(ia + H + kk) : make_float2(0.f, 0.f);
        if (k > N / 2) {
            A.y = -A.y;
            B.y = -B.y;
        }
        // conj(Z) for the inverse through the forward transform
        v[m] = make_float2(A.x - B.y, -(A.y + B.x));
    }
    fft_regs<N, RF_E, G::WS>(v, t, buf, tw);
    const float sc = 1.0f / (float)N;
    float* oa = out + la * N + t;
#pragma unroll
    for (int m = 0; m < RF_E; ++m) {
        // z = conj(v) / n: a = Re z, b = Im z
        if (ok0) __stcs(oa + m * T, v[m].x * sc);
        if (ok1) __stcs(oa + N + m * T, -v[m].y * sc);
    }
}

struct RfKernels {
    int n, lines, threads, smem;
    cudaError_t (*prepare)();
    void (*r2c)(dim3, cudaStream_t, const float*, float2*, long long, const float2*);
    void (*c2r)(dim3, cudaStream_t, const float2*, float*, long long, const float2*);
};

template <int N>
cudaError_t rf_prepare() {
    cudaError_t e = cudaFuncSetAttribute(k_r2c<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, RfGeom<N>::SMEM);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_c2r<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, RfGeom<N>::SMEM);
}
template <int N>
void rf_r2c(dim3 g, cudaStream_t s, const float* in, float2* out, long long batch, const float2* tw) {
    k_r2c<N><<<g, RfGeom<N>::THREADS, RfGeom<N>::SMEM, s>>>(in, out, batch, tw);
}
template <int N>
void rf_c2r(dim3 g, cudaStream_t s, const float2* in, float* out, long long batch, const float2* tw) {
    k_c2r<N><<<g, RfGeom<N>::THREADS, RfGeom<N>::SMEM, s>>>(in, out, batch, tw);
}

#define MFFT_RF(N) {N, RfGeom<N>::LINES, RfGeom<N>::THREADS, RfGeom<N>::SMEM, &rf_prepare<N>, &rf_r2c<N>, &rf_c2r<N>}
const RfKernels g_rf[] = {MFFT_RF(64),   MFFT_RF(128),  MFFT_RF(256),  MFFT_RF(512), MFFT_RF(1024),
                          MFFT_RF(2048), MFFT_RF(4096), MFFT_RF(8192), MFFT_RF(16384)};

const RfKernels* find_rf(int64_t n) {
    for (const auto& k : g_rf)
        if (k.n == n) return &k;
    return nullptr;
}

int real_exec(mfft_plan* plan, const void* in, void* out, int64_t batch, int flags, void* stream, bool forward) {
    if (!plan) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    if (batch < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, batch, -1, "batch must be >= 0");
    if (flags != MFFT_HOST_MEMORY && flags != MFFT_DEVICE_MEMORY)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown flags %d", flags);
    if (batch > 0 && (!in || !out)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL buffer");
    const RfKernels* k = find_rf(plan->n);
    if (!k)
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, plan->n, -1, -1,
                         "real-input FFT sizes are powers of two 64..16384, got %lld", (long long)plan->n);
    if (batch == 0) return MFFT_SUCCESS;
    if (((batch + 1) / 2 + k->lines - 1) / k->lines > 0x7fffffffLL)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, batch, -1, "batch too large");
    DeviceGuard g(plan->ctx->device);
    cudaError_t e = k->prepare();  // shared-memory opt-in on the current device
    if (e != cudaSuccess) return cuda_error(e, "real FFT kernel attributes");
    const float2* tw = plan->line.tw;  // the plan's E = 16 twiddle rows for n
    if (!tw || plan->line.k->e != 16) {
        float2* t2 = nullptr;
        int st = line_twiddles(plan->ctx, (int)plan->n, &t2);
        if (st) return st;
        tw = t2;
    }
    const size_t real_line = (size_t)plan->n * sizeof(float);
    const size_t cplx_line = (size_t)(plan->n / 2 + 1) * sizeof(float2);
    auto body = [&](const void* di, void* dout, int64_t nl, cudaStream_t s) -> int {
        const long long ctas = ((nl + 1) / 2 + k->lines - 1) / k->lines;
        if (forward) k->r2c(dim3((unsigned)ctas), s, (const float*)di, (float2*)dout, nl, tw);
        else k->c2r(dim3((unsigned)ctas), s, (const float2*)di, (float*)dout, nl, tw);
        cudaError_t le = cudaGetLastError();
        return le == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(le, "real FFT launch");
    };
    if (flags == MFFT_DEVICE_MEMORY) return body(in, out, batch, (cudaStream_t)stream);
    // line pairs share a transform, so chunks start on even lines
    return run_host_lines(plan->ctx, in, out, batch, forward ? real_line : cplx_line,
                          forward ? cplx_line : real_line, body, false, true);
}

}  // namespace

}  // namespace mfft

extern "C" int mfft_exec_r2c(mfft_plan* plan, const float* in, void* out, int64_t batch, int flags, void* stream) {
    return mfft::real_exec(plan, in, out, batch, flags, stream, true);
}

extern "C" int mfft_exec_c2r(mfft_plan* plan, const void* in, float* out, int64_t batch, int flags, void* stream) {
    return mfft::real_exec(plan, in, out, batch, flags, stream, false);
}
