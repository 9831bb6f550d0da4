// noalloc.cu -- mfft_fourstep_noalloc: the four-step FFT (n = 2^15 .. 2^20)
// for callers that cannot allocate device memory.
//
// Some callers can't call cudaMalloc: code running under an external memory
// budget that owns every device allocation (a framework's caching allocator,
// a real-time or embedded host that reserves memory once at start-up), or a
// plug-in host that forbids its plug-ins from allocating.  mfft_plan_create
// allocates (twiddle tables and a 128 MiB intermediate buffer), so those
// callers get this entry point instead: it takes device input and output
// pointers and allocates nothing.  Its intermediate buffer and its twiddle
// tables are file-scope __device__ arrays of fixed size, reserved on every
// GPU that loads this code and held until the process exits:
//   - intermediate: NOALLOC_SCRATCH_POINTS = 2^21 complex64 (16 MiB); a
//     batch is processed in chunks of 2^21 / n lines, so any batch works;
//   - tables: about 100 KB.
// Every call shares these arrays and leaves the last call's data in the
// intermediate.  Nothing needs to start at zero (the column pass overwrites
// every element the row pass reads), but two calls that overlap on the GPU
// (different streams, or different host threads) race on the intermediate:
// serialise them.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "capi_internal.h"
#include "stockham.cuh"

namespace mfft {
namespace {

constexpr long long NOALLOC_SCRATCH_POINTS = 1LL << 21;
constexpr int NA_TILE = 16;       // rows per row-pass CTA, columns per column-pass CTA
constexpr int NA_FINE = 1024;
constexpr int NA_LINE_TW = 640;   // >= SPlan<L,16>::TWSIZE for L = 128 .. 1024
constexpr int NA_SIZES = 6;       // n = 2^15 .. 2^20

static __device__ __align__(256) float2 g_noalloc_scratch[NOALLOC_SCRATCH_POINTS];
static __device__ __align__(256) float2 g_noalloc_line_tw[4][NA_LINE_TW];  // L = 128, 256, 512, 1024
static __device__ __align__(256) float2 g_noalloc_fine[NA_SIZES][NA_FINE];
static __device__ __align__(256) float2 g_noalloc_coarse[NA_SIZES][NA_FINE];

struct NoallocDevice {
    bool ready = false;
    unsigned long long ctx_id = 0;  // the CUDA context the addresses and tables belong to
    float2* scratch = nullptr;
    float2* line_tw = nullptr;
    float2* fine = nullptr;
    float2* coarse = nullptr;
};
std::mutex g_noalloc_mu;
NoallocDevice g_noalloc_dev[64];

__host__ __device__ constexpr int na_tile_cols(int L) { return L >= 1024 ? 8 : NA_TILE; }

// Every launch of this file goes through here and is checked as it is made:
// the status is this launch's own, so an earlier error of unrelated code is
// neither reported as ours nor cleared.
template <class... KArgs, class... Args>
cudaError_t na_launch(void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                      Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    return cudaLaunchKernelEx(&cfg, k, (KArgs)args...);
}

__global__ void k_na_line_rows(float2* tw, int off, int ns, int radix, int rowlen) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ns * rowlen) return;
    int k = idx / rowlen, e = idx % rowlen;
    double s, c;
    sincospi(-2.0 * (double)((1 << e) * k) / (double)(ns * radix), &s, &c);
    tw[off + idx] = make_float2((float)c, (float)s);
}

__global__ void k_na_tables(float2* fine, float2* coarse, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s, c;
    if (i < NA_FINE) {
        sincospi(-2.0 * (double)i / (double)n, &s, &c);
        fine[i] = make_float2((float)c, (float)s);
    }
    if (i < n / NA_FINE) {
        sincospi(-2.0 * (double)i * NA_FINE / (double)n, &s, &c);
        coarse[i] = make_float2((float)c, (float)s);
    }
}

template <int L>
cudaError_t na_gen_line(float2* tw, cudaStream_t s) {
    using PL = SPlan<L, 16>;
    static_assert(PL::TWSIZE <= NA_LINE_TW, "line twiddle slot too small");
    for (int p = 1; p < PL::NPASS; ++p) {
        int cnt = PL::span(p) * PL::twrow(PL::radix(p));
        cudaError_t e = na_launch(k_na_line_rows, (unsigned)((cnt + 255) / 256), 256u, 0, s, tw, PL::twoff(p),
                                  PL::span(p), PL::radix(p), PL::twrow(PL::radix(p)));
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// column pass: C columns per CTA, FFT of length L down each column, times
// W_N^{col*k1}, written to the same positions of the intermediate.
template <int L, bool INV>
__global__ void __launch_bounds__(L / 16 * na_tile_cols(L))
    k_na_cols(const float2* __restrict__ in, float2* __restrict__ mid, int n2, const float2* __restrict__ tw,
              const float2* __restrict__ fine, const float2* __restrict__ coarse) {
    constexpr int E = 16, T = L / E, C = na_tile_cols(L);
    extern __shared__ float2 smem[];
    const int tiles = n2 / C;
    const long long b = blockIdx.x / tiles;
    const int c = threadIdx.x % C;
    const int col = (blockIdx.x % tiles) * C + c;
    const int t = threadIdx.x / C;
    const size_t N = (size_t)L * n2;
    const float2* src = in + b * N + col;
    float2 v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        v[m] = __ldcs(src + (size_t)(t + m * T) * n2);
        if constexpr (INV) v[m].y = -v[m].y;
    }
    fft_regs<L, E, false>(v, t, ColLine<C>{smem, c}, tw);
    float2* dst = mid + b * N + col;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const unsigned k1 = (unsigned)(t + m * T);
        const unsigned e = (unsigned)col * k1;
        const float2 w = cmul(__ldg(fine + (e & (NA_FINE - 1))), __ldg(coarse + (e >> 10)));
        dst[(size_t)k1 * n2] = cmul(v[m], w);
    }
}

// row pass: 16 rows per CTA, FFT of length L along each row, result
// X[k1 + n1*k2] stored at out[k2*n1 + k1].
template <int L, bool INV>
__global__ void __launch_bounds__(L) k_na_rows(const float2* __restrict__ mid, float2* __restrict__ out, int n1,
                                               const float2* __restrict__ tw) {
    constexpr int E = 16, T = L / E, RW = NA_TILE;
    extern __shared__ float2 smem[];
    const int groups = n1 / RW;
    const long long b = blockIdx.x / groups;
    const int row0 = (blockIdx.x % groups) * RW;
    const size_t N = (size_t)n1 * L;
    const float4* src = reinterpret_cast<const float4*>(mid + b * N + (size_t)row0 * L);
    for (int q = threadIdx.x; q < RW * L / 2; q += L) {
        const float4 x = src[q];
        const int e = 2 * q, r = e / L, i = e % L;
        SwzLine<RW> line{smem, r};
        line[i] = make_float2(x.x, x.y);
        line[i + 1] = make_float2(x.z, x.w);
    }
    __syncthreads();
    const int r = threadIdx.x % RW;
    const int t = threadIdx.x / RW;
    const SwzLine<RW> line{smem, r};
    float2 v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = line[t + m * T];
    __syncthreads();
    fft_regs<L, E, false>(v, t, line, tw);
    float2* dst = out + b * N + row0 + r;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        float2 y = v[m];
        if constexpr (INV) {
            const float s = 1.0f / (float)N;
            y = make_float2(y.x * s, -y.y * s);
        }
        __stcs(dst + (size_t)(t + m * T) * n1, y);
    }
}

template <int L>
cudaError_t na_prepare() {
    const int cs = L * na_tile_cols(L) * (int)sizeof(float2);
    const int rs = L * NA_TILE * (int)sizeof(float2);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_na_cols<L, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, cs))) return e;
    if ((e = cudaFuncSetAttribute(k_na_cols<L, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, cs))) return e;
    if ((e = cudaFuncSetAttribute(k_na_rows<L, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, rs))) return e;
    return cudaFuncSetAttribute(k_na_rows<L, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, rs);
}

template <int L>
cudaError_t na_cols(const float2* in, float2* mid, int n2, const float2* tw, const float2* fine,
                    const float2* coarse, long long nb, bool inv, cudaStream_t s) {
    constexpr int C = na_tile_cols(L);
    const size_t smem = (size_t)L * C * sizeof(float2);
    const unsigned blocks = (unsigned)(nb * (n2 / C));
    return inv ? na_launch(k_na_cols<L, true>, blocks, (unsigned)(L / 16 * C), smem, s, in, mid, n2, tw, fine, coarse)
               : na_launch(k_na_cols<L, false>, blocks, (unsigned)(L / 16 * C), smem, s, in, mid, n2, tw, fine, coarse);
}

template <int L>
cudaError_t na_rows(const float2* mid, float2* out, int n1, const float2* tw, long long nb, bool inv,
                    cudaStream_t s) {
    const size_t smem = (size_t)L * NA_TILE * sizeof(float2);
    const unsigned blocks = (unsigned)(nb * (n1 / NA_TILE));
    return inv ? na_launch(k_na_rows<L, true>, blocks, (unsigned)L, smem, s, mid, out, n1, tw)
               : na_launch(k_na_rows<L, false>, blocks, (unsigned)L, smem, s, mid, out, n1, tw);
}

// Unique id of the calling thread's current CUDA context (the device's primary
// context, made current if no context is).  A device reset destroys the
// primary context; the next one gets a new id, so the set-up below is redone
// for it instead of reusing addresses and tables of the old context.
// (driver entry points through the runtime: the library has no link-time
// dependency on the driver library)
int na_context_id(int dev, unsigned long long* id) {
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f);
    });
    if (!get_current || !get_id)
        return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "no-alloc set-up: driver context queries unavailable");
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || !c) {
        cudaError_t e = cudaSetDevice(dev);  // initialises and binds the primary context
        if (e != cudaSuccess) return cuda_error(e, "no-alloc set-up: cudaSetDevice");
        if (get_current(&c) != CUDA_SUCCESS || !c)
            return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "no-alloc set-up: no current CUDA context");
    }
    if (get_id(c, id) != CUDA_SUCCESS)
        return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "no-alloc set-up: cuCtxGetId failed");
    return MFFT_SUCCESS;
}

// Once per device (and again after a device reset), with that device
// current: resolve the arrays' device addresses (cudaGetSymbolAddress), fill
// the tables and raise the kernels' shared-memory limits.  Launches kernels
// but allocates nothing.
int na_setup(int dev, cudaStream_t s, NoallocDevice** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocDevice& d = g_noalloc_dev[dev];
    unsigned long long id = 0;
    int st = na_context_id(dev, &id);
    if (st) return st;
    if (d.ready && d.ctx_id == id) {
        *out = &d;
        return MFFT_SUCCESS;
    }
    d.ready = false;
    cudaError_t e = cudaGetSymbolAddress((void**)&d.scratch, g_noalloc_scratch);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&d.line_tw, g_noalloc_line_tw);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&d.fine, g_noalloc_fine);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&d.coarse, g_noalloc_coarse);
    if (e != cudaSuccess) return cuda_error(e, "no-alloc set-up: cudaGetSymbolAddress");
    if ((e = na_prepare<128>()) || (e = na_prepare<256>()) || (e = na_prepare<512>()) ||
        (e = na_prepare<1024>()))
        return cuda_error(e, "no-alloc set-up: kernel attributes");
    if ((e = na_gen_line<128>(d.line_tw + 0 * NA_LINE_TW, s)) || (e = na_gen_line<256>(d.line_tw + 1 * NA_LINE_TW, s)) ||
        (e = na_gen_line<512>(d.line_tw + 2 * NA_LINE_TW, s)) || (e = na_gen_line<1024>(d.line_tw + 3 * NA_LINE_TW, s)))
        return cuda_error(e, "no-alloc set-up: twiddle launch");
    for (int i = 0; i < NA_SIZES; ++i) {
        e = na_launch(k_na_tables, (unsigned)((NA_FINE + 255) / 256), 256u, 0, s, d.fine + i * NA_FINE,
                      d.coarse + i * NA_FINE, 1 << (15 + i));
        if (e != cudaSuccess) return cuda_error(e, "no-alloc set-up: twiddle launch");
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "no-alloc set-up: tables");
    d.ctx_id = id;
    d.ready = true;
    *out = &d;
    return MFFT_SUCCESS;
}

int na_line_slot(int L) { return L == 128 ? 0 : L == 256 ? 1 : L == 512 ? 2 : 3; }

}  // namespace
}  // namespace mfft

// Four-step C2C FFT of `batch` lines of length n (a power of two from 2^15 to
// 2^20) on device memory, enqueued on `stream`; no device memory is allocated.
// The first call on a device does a one-time set-up that launches kernels and
// waits for them: make that first call before any stream capture begins.  The
// set-up is redone on the first call after a device reset.
extern "C" int mfft_fourstep_noalloc(const void* in, void* out, int64_t n, int64_t batch, int direction,
                                     void* stream) {
    using namespace mfft;
    if (!is_pow2_in(n, 1 << 15, 1 << 20))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, n, -1, -1,
                         "mfft_fourstep_noalloc: n=%lld unsupported; it takes powers of two from 32768 to "
                         "1048576 (its intermediate holds %lld complex values)",
                         (long long)n, (long long)NOALLOC_SCRATCH_POINTS);
    if (batch < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, batch, -1, "batch must be >= 0");
    if (direction != MFFT_FORWARD && direction != MFFT_INVERSE)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "direction must be -1 or +1, got %d", direction);
    if (batch == 0) return MFFT_SUCCESS;
    if (!in || !out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL buffer");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "No CUDA device available");
    cudaStream_t s = (cudaStream_t)stream;
    NoallocDevice* d = nullptr;
    int st = na_setup(dev, s, &d);
    if (st) return st;

    const int m = ilog2c(n);
    const int n1 = 1 << (m / 2), n2 = (int)(n / n1);
    const float2* ctw = d->line_tw + na_line_slot(n1) * NA_LINE_TW;
    const float2* rtw = d->line_tw + na_line_slot(n2) * NA_LINE_TW;
    const float2* fine = d->fine + (m - 15) * NA_FINE;
    const float2* coarse = d->coarse + (m - 15) * NA_FINE;
    const bool inv = (direction == MFFT_INVERSE);
    const long long chunk = NOALLOC_SCRATCH_POINTS / n;
    const float2* x = (const float2*)in;
    float2* y = (float2*)out;
    for (int64_t b0 = 0; b0 < batch; b0 += chunk) {
        const long long nb = batch - b0 < chunk ? batch - b0 : chunk;
        switch (n1) {
            case 128: e = na_cols<128>(x + b0 * n, d->scratch, n2, ctw, fine, coarse, nb, inv, s); break;
            case 256: e = na_cols<256>(x + b0 * n, d->scratch, n2, ctw, fine, coarse, nb, inv, s); break;
            case 512: e = na_cols<512>(x + b0 * n, d->scratch, n2, ctw, fine, coarse, nb, inv, s); break;
            default: e = na_cols<1024>(x + b0 * n, d->scratch, n2, ctw, fine, coarse, nb, inv, s); break;
        }
        if (e != cudaSuccess) return cuda_error(e, "mfft_fourstep_noalloc column-pass launch");
        switch (n2) {
            case 256: e = na_rows<256>(d->scratch, y + b0 * n, n1, rtw, nb, inv, s); break;
            case 512: e = na_rows<512>(d->scratch, y + b0 * n, n1, rtw, nb, inv, s); break;
            default: e = na_rows<1024>(d->scratch, y + b0 * n, n1, rtw, nb, inv, s); break;
        }
        if (e != cudaSuccess) return cuda_error(e, "mfft_fourstep_noalloc row-pass launch");
    }
    return MFFT_SUCCESS;
}
