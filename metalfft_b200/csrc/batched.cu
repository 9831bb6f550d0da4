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
#include "pdl.cuh"
#include "stockham.cuh"
#include "tma.cuh"

namespace mfft {

__global__ void k_twiddle_rows(float2* tw, int off, int ns, int radix, int rowlen) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ns * rowlen) return;
    int k = idx / rowlen, e = idx % rowlen;
    double s, c;
    sincospi(-2.0 * (double)((1 << e) * k) / (double)(ns * radix), &s, &c);
    tw[off + idx] = make_float2((float)c, (float)s);
}


// Streams a thread's E results to dst[m*T]: the inverse conjugates and scales
// by 1/N (MetalFFT.swift:56-65); adj (the adjoint of the transform) drops that
// scale from the inverse and puts it on the forward.  Power-of-two scalings
// are exact, so the adjoint of the forward is exactly N x inverse.
template <int N, int E, bool INV>
__device__ __forceinline__ void store_line(float2* dst, const float2 (&v)[E], int adj) {
    constexpr int T = N / E;
    if constexpr (INV) {
        const float s = adj ? 1.0f : 1.0f / (float)N;
#pragma unroll
        for (int m = 0; m < E; ++m) __stcs(dst + m * T, make_float2(v[m].x * s, -v[m].y * s));
    } else if (adj) {
        const float s = 1.0f / (float)N;
#pragma unroll
        for (int m = 0; m < E; ++m) __stcs(dst + m * T, make_float2(v[m].x * s, v[m].y * s));
    } else {
#pragma unroll
        for (int m = 0; m < E; ++m) __stcs(dst + m * T, v[m]);
    }
}

template <int N, int E, int FPB, bool INV>
__global__ void __launch_bounds__(SPlan<N, E>::T * FPB)
    k_fft_batched(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
                  const float2* __restrict__ tw, int adj) {
    constexpr int T = SPlan<N, E>::T;
    constexpr bool WS = (T <= 32);
    extern __shared__ float2 smem[];
    const int lf = threadIdx.x / T;
    const int t = threadIdx.x % T;
    const long long f = (long long)blockIdx.x * FPB + lf;
    const bool ok = f < batch;
    const PadLineS buf{smem + lf * spad_size(N)};
    float2 v[E];
    grid_dep_wait();
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
    if (ok) store_line<N, E, INV>(out + (size_t)f * N + t, v, adj);
}

template <int N, int E, int FPB, bool INV>
static cudaError_t launch_batched(const float2* in, float2* out, long long batch, const float2* tw,
                                  int*, cudaStream_t s, int adj) {
    constexpr int threads = SPlan<N, E>::T * FPB;
    constexpr int smem = FPB * spad_size(N) * (int)sizeof(float2);
    long long blocks = (batch + FPB - 1) / FPB;
    if (blocks <= 0) return cudaSuccess;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    return launch_pdl(k_fft_batched<N, E, FPB, INV>, (unsigned)blocks, threads, smem, s, in, out, batch, tw, adj);
}

template <class K>
static cudaError_t set_smem_attrs(K kernel, int smem) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
}

template <int N, int E, int FPB>
static cudaError_t prepare_batched() {
    constexpr int smem = FPB * spad_size(N) * (int)sizeof(float2);
    cudaError_t e = set_smem_attrs(k_fft_batched<N, E, FPB, false>, smem);
    if (e != cudaSuccess) return e;
    return set_smem_attrs(k_fft_batched<N, E, FPB, true>, smem);
}

// ---- persistent variant: TMA bulk prefetch of the next line groups ---------
//
// Each CTA walks line groups g = blockIdx.x, blockIdx.x + gridDim.x, ... (a
// group is FPB consecutive lines, one contiguous chunk of memory).  Thread 0
// keeps STAGES groups in flight with 1-D cp.async.bulk copies into the stage
// buffers; the CTA waits on the stage's mbarrier (bounded), reads its values
// into registers, reuses the same stage buffer (padded) for the exchanges,
// hands the buffer back to the copy engine for group g + STAGES*gridDim.x and
// stores its results.  Global loads never stall the compute warps.
template <int N, int E, int FPB, int STAGES, bool INV>
__global__ void __launch_bounds__(SPlan<N, E>::T * FPB)
    k_fft_stream(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
                 const float2* __restrict__ tw, int* dev_err, int adj) {
    constexpr int T = SPlan<N, E>::T;
    constexpr bool WS = (T <= 32);
    constexpr int STAGE = FPB * spad_size(N);  // float2 per stage buffer
    extern __shared__ __align__(128) float2 smem[];
    __shared__ __align__(8) uint64_t full[STAGES];
    const long long groups = (batch + FPB - 1) / FPB;
    const int lf = threadIdx.x / T;
    const int t = threadIdx.x % T;

    auto issue = [&](long long g, int s) {
        long long lines = batch - g * FPB;
        if (lines > FPB) lines = FPB;
        const uint32_t bytes = (uint32_t)(lines * N * sizeof(float2));
        mbar_arrive_expect_tx(&full[s], bytes);
        bulk_g2s(smem + s * STAGE, in + (size_t)g * FPB * N, bytes, &full[s]);
    };

    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
        fence_proxy_async_smem();
    }
    grid_dep_wait();  // every thread: the previous kernel's writes are visible
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) {
            const long long g = blockIdx.x + (long long)s * gridDim.x;
            if (g < groups) issue(g, s);
        }
    }
    __syncthreads();

    int it = 0;
    for (long long g = blockIdx.x; g < groups; g += gridDim.x, ++it) {
        const int s = it % STAGES;
        const uint32_t parity = (uint32_t)((it / STAGES) & 1);
        // Every thread waits (bounded) on its own; a thread that gives up still
        // reaches the barrier below, which takes the decision for the whole CTA,
        // so no thread leaves while another waits at a barrier.
        const bool landed = mbar_wait(&full[s], parity);
        float2* buf = smem + s * STAGE;
        const long long f = g * FPB + lf;
        const bool ok = f < batch;
        float2 v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            v[m] = ok ? buf[lf * N + t + m * T] : make_float2(0.f, 0.f);
            if constexpr (INV) v[m].y = -v[m].y;
        }
        // the raw group is in registers; the buffer becomes the exchange area
        if (__syncthreads_or(!landed)) {
            if (threadIdx.x == 0) {
                report_device_error(dev_err, DEV_ERR_TMA_TIMEOUT);
                // copies still in flight land before the CTA's shared memory goes away
#pragma unroll
                for (int d = 0; d < STAGES; ++d) {
                    const int it2 = it + d;
                    if (g + (long long)d * gridDim.x < groups)
                        mbar_wait(&full[it2 % STAGES], (uint32_t)((it2 / STAGES) & 1));
                }
            }
            return;
        }
        fft_regs<N, E, WS>(v, t, PadLineS{buf + lf * spad_size(N)}, tw);
        fence_proxy_async_smem();  // order this thread's exchange writes before the next bulk copy
        __syncthreads();           // every exchange access of this buffer is done
        if (threadIdx.x == 0) {
            const long long gn = g + (long long)STAGES * gridDim.x;
            if (gn < groups) issue(gn, s);
        }
        if (ok) store_line<N, E, INV>(out + (size_t)f * N + t, v, adj);
    }
}

static int device_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

template <int N, int E, int FPB, int STAGES, bool INV>
static cudaError_t launch_stream(const float2* in, float2* out, long long batch, const float2* tw,
                                 int* dev_err, cudaStream_t s, int adj) {
    constexpr int threads = SPlan<N, E>::T * FPB;
    constexpr int smem = STAGES * FPB * spad_size(N) * (int)sizeof(float2);
    static int occ = 0;
    if (!occ) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fft_stream<N, E, FPB, STAGES, INV>, threads,
                                                      smem);
        if (occ <= 0) occ = 1;
    }
    const long long groups = (batch + FPB - 1) / FPB;
    if (groups <= 0) return cudaSuccess;
    long long blocks = (long long)device_sms() * occ;
    if (blocks > groups) blocks = groups;
    return launch_pdl(k_fft_stream<N, E, FPB, STAGES, INV>, (unsigned)blocks, threads, smem, s, in, out, batch, tw,
                      dev_err, adj);
}

template <int N, int E, int FPB, int STAGES>
static cudaError_t prepare_stream() {
    constexpr int smem = STAGES * FPB * spad_size(N) * (int)sizeof(float2);
    cudaError_t e = set_smem_attrs(k_fft_stream<N, E, FPB, STAGES, false>, smem);
    if (e != cudaSuccess) return e;
    return set_smem_attrs(k_fft_stream<N, E, FPB, STAGES, true>, smem);
}

template <int N, int E>
static void gen_tw(float2* tw, cudaStream_t s) {
    gen_twiddles<N, E>(tw, s);
}

#define MFFT_BATCHED(N, E, FPB)                                                            \
    {N,                                                                                    \
     E,                                                                                    \
     FPB,                                                                                  \
     0,                                                                                    \
     SPlan<N, E>::T * FPB,                                                                 \
     FPB * spad_size(N) * (int)sizeof(float2),                                             \
     SPlan<N, E>::TWSIZE,                                                                  \
     &launch_batched<N, E, FPB, false>,                                                    \
     &launch_batched<N, E, FPB, true>,                                                     \
     &prepare_batched<N, E, FPB>,                                                          \
     &gen_tw<N, E>}

#define MFFT_STREAM(N, E, FPB, ST)                                                         \
    {N,                                                                                    \
     E,                                                                                    \
     FPB,                                                                                  \
     ST,                                                                                   \
     SPlan<N, E>::T * FPB,                                                                 \
     ST * FPB * spad_size(N) * (int)sizeof(float2),                                        \
     SPlan<N, E>::TWSIZE,                                                                  \
     &launch_stream<N, E, FPB, ST, false>,                                                 \
     &launch_stream<N, E, FPB, ST, true>,                                                  \
     &prepare_stream<N, E, FPB, ST>,                                                       \
     &gen_tw<N, E>}

static const BatchedKernel g_batched[] = {
    // persistent, TMA-prefetched (stages = groups in flight per CTA)
    MFFT_STREAM(64, 16, 64, 2), MFFT_STREAM(128, 16, 32, 2), MFFT_STREAM(256, 16, 16, 2),
    MFFT_STREAM(512, 16, 8, 2), MFFT_STREAM(1024, 16, 4, 2), MFFT_STREAM(2048, 16, 2, 2),
    MFFT_STREAM(4096, 16, 1, 2), MFFT_STREAM(4096, 16, 1, 3), MFFT_STREAM(4096, 16, 2, 2),
    MFFT_STREAM(4096, 8, 1, 2), MFFT_STREAM(8192, 16, 1, 2), MFFT_STREAM(8192, 8, 1, 2),
    MFFT_STREAM(2048, 16, 1, 3), MFFT_STREAM(1024, 16, 2, 3),
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

const BatchedKernel* find_batched(int n, int e, int fpb, int stages) {
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    for (int i = 0; i < cnt; ++i)
        if (ks[i].n == n && ks[i].e == e && ks[i].fpb == fpb && ks[i].stages == stages) return &ks[i];
    return nullptr;
}

// Default choice before autotuning: the fastest variant of a B200 sweep at
// 512 MiB per buffer (fraction of the measured 6555 GB/s copy bandwidth):
// 64: 0.87, 256: 0.87, 1024: 0.92, 2048: 0.90, 4096: 0.86, 8192: 0.58,
// 16384: 0.45.  Sizes without a sweep entry take E = 16 near 256 threads.
const BatchedKernel* default_batched(int n) {
    static const int pref[][4] = {{64, 16, 64, 2},  {128, 16, 32, 2},  {256, 8, 8, 0},
                                  {512, 16, 8, 2},  {1024, 16, 2, 3},  {2048, 16, 1, 3},
                                  {4096, 16, 1, 2}, {8192, 16, 1, 2},  {16384, 16, 1, 0}};
    for (const auto& p : pref)
        if (p[0] == n) {
            const BatchedKernel* k = find_batched(p[0], p[1], p[2], p[3]);
            if (k) return k;
        }
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    const BatchedKernel* best = nullptr;
    for (int i = 0; i < cnt; ++i) {
        if (ks[i].n != n || ks[i].e != 16 || ks[i].stages != 0) continue;
        if (!best || abs(ks[i].threads - 256) < abs(best->threads - 256)) best = &ks[i];
    }
    return best;
}

}  // namespace mfft
