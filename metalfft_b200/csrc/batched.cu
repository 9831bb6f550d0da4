// batched.cu -- batched C2C FFT kernels for N = 64 .. 16384 (one line per T
// threads, FPB lines per CTA) and their registry.
//
// B200 form of MetalFFT.forward(batch:) -> dispatchBatch
// (Sources/MetalFFT/FFT/MetalFFT.swift:108-133,159-204), which launches one
// threadgroup per line of fft_4096_batched / fft_N_stockham
// (Sources/MetalFFT/Resources/fft_4096_batched.metal:79-203,
//  fft_multisize.metal:62-687).  Here small lines share a CTA (FPB > 1) so
// every CTA has >= 128 threads, loads and stores are streaming (.cs) and
// coalesced, and the inverse's conjugations and 1/N scale
// (MetalFFT.swift:56-65) are fused into the load and the store.
#include "kernels.h"
#include "stockham.cuh"

namespace mfft {

__global__ void k_twiddle_rows(float2* tw, int off, int ns, int radix) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ns * radix) return;
    int k = idx / radix, r = idx % radix;
    double s, c;
    sincospi(-2.0 * (double)(r * k) / (double)(ns * radix), &s, &c);
    tw[off + idx] = make_float2((float)c, (float)s);
}

template <int N, int E, int FPB, bool INV>
__global__ void __launch_bounds__(SPlan<N, E>::T * FPB)
    k_fft_batched(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
                  const float2* __restrict__ tw) {
    constexpr int T = SPlan<N, E>::T;
    constexpr bool WS = (T <= 32);
    extern __shared__ float2 smem[];
    const int lf = threadIdx.x / T;
    const int t = threadIdx.x % T;
    const long long f = (long long)blockIdx.x * FPB + lf;
    const bool ok = f < batch;
    const PadLine buf{smem + lf * spad_size(N)};
    float2 v[E];
    if (ok) {
        const float2* src = in + (size_t)f * N + t;
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = __ldcs(src + m * T);
    } else {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = make_float2(0.f, 0.f);
    }
    if constexpr (INV) {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m].y = -v[m].y;
    }
    fft_regs<N, E, WS>(v, t, buf, tw);
    if (ok) {
        float2* dst = out + (size_t)f * N + t;
        if constexpr (INV) {
            const float s = 1.0f / (float)N;
#pragma unroll
            for (int m = 0; m < E; ++m) __stcs(dst + m * T, make_float2(v[m].x * s, -v[m].y * s));
        } else {
#pragma unroll
            for (int m = 0; m < E; ++m) __stcs(dst + m * T, v[m]);
        }
    }
}

template <int N, int E, int FPB, bool INV>
static cudaError_t launch_batched(const float2* in, float2* out, long long batch, const float2* tw,
                                  cudaStream_t s) {
    constexpr int threads = SPlan<N, E>::T * FPB;
    constexpr int smem = FPB * spad_size(N) * (int)sizeof(float2);
    long long blocks = (batch + FPB - 1) / FPB;
    if (blocks <= 0) return cudaSuccess;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    k_fft_batched<N, E, FPB, INV><<<(unsigned)blocks, threads, smem, s>>>(in, out, batch, tw);
    return cudaGetLastError();
}

template <int N, int E, int FPB>
static cudaError_t prepare_batched() {
    constexpr int smem = FPB * spad_size(N) * (int)sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(k_fft_batched<N, E, FPB, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_fft_batched<N, E, FPB, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <int N, int E>
static void gen_tw(float2* tw, cudaStream_t s) {
    gen_twiddles<N, E>(tw, s);
}

#define MFFT_BATCHED(N, E, FPB)                                                            \
    {N,                                                                                    \
     E,                                                                                    \
     FPB,                                                                                  \
     SPlan<N, E>::T * FPB,                                                                 \
     FPB * spad_size(N) * (int)sizeof(float2),                                             \
     SPlan<N, E>::TWSIZE,                                                                  \
     &launch_batched<N, E, FPB, false>,                                                    \
     &launch_batched<N, E, FPB, true>,                                                     \
     &prepare_batched<N, E, FPB>,                                                          \
     &gen_tw<N, E>}

static const BatchedKernel g_batched[] = {
    // E = 16: radix-16 passes (+ a radix 2/4/8 tail)
    MFFT_BATCHED(64, 16, 32), MFFT_BATCHED(64, 16, 64), MFFT_BATCHED(64, 16, 128),
    MFFT_BATCHED(128, 16, 16), MFFT_BATCHED(128, 16, 32), MFFT_BATCHED(128, 16, 64),
    MFFT_BATCHED(256, 16, 8), MFFT_BATCHED(256, 16, 16), MFFT_BATCHED(256, 16, 32),
    MFFT_BATCHED(512, 16, 4), MFFT_BATCHED(512, 16, 8), MFFT_BATCHED(512, 16, 16),
    MFFT_BATCHED(1024, 16, 2), MFFT_BATCHED(1024, 16, 4), MFFT_BATCHED(1024, 16, 8),
    MFFT_BATCHED(2048, 16, 1), MFFT_BATCHED(2048, 16, 2), MFFT_BATCHED(2048, 16, 4),
    MFFT_BATCHED(4096, 16, 1), MFFT_BATCHED(4096, 16, 2),
    MFFT_BATCHED(8192, 16, 1),
    MFFT_BATCHED(16384, 16, 1),
    // E = 8: radix-8 passes (+ tail), twice the threads per line
    MFFT_BATCHED(64, 8, 16), MFFT_BATCHED(64, 8, 32),
    MFFT_BATCHED(128, 8, 8), MFFT_BATCHED(128, 8, 16),
    MFFT_BATCHED(256, 8, 4), MFFT_BATCHED(256, 8, 8),
    MFFT_BATCHED(512, 8, 2), MFFT_BATCHED(512, 8, 4),
    MFFT_BATCHED(1024, 8, 1), MFFT_BATCHED(1024, 8, 2),
    MFFT_BATCHED(2048, 8, 1),
    MFFT_BATCHED(4096, 8, 1),
    MFFT_BATCHED(8192, 8, 1),
};

const BatchedKernel* batched_kernels(int* count) {
    *count = (int)(sizeof(g_batched) / sizeof(g_batched[0]));
    return g_batched;
}

const BatchedKernel* find_batched(int n, int e, int fpb) {
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    for (int i = 0; i < cnt; ++i)
        if (ks[i].n == n && ks[i].e == e && ks[i].fpb == fpb) return &ks[i];
    return nullptr;
}

// Default choice before autotuning: E = 16 and the CTA closest to 256 threads.
const BatchedKernel* default_batched(int n) {
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    const BatchedKernel* best = nullptr;
    for (int i = 0; i < cnt; ++i) {
        if (ks[i].n != n || ks[i].e != 16) continue;
        if (!best || abs(ks[i].threads - 256) < abs(best->threads - 256)) best = &ks[i];
    }
    return best;
}

}  // namespace mfft
