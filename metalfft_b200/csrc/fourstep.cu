// fourstep.cu -- C2C FFT for N = 2^15 .. 2^20 as N = n1 * n2 (both <= 1024).
//
// B200 form of the reference's four-step plan (dispatchFourStep,
// Sources/MetalFFT/FFT/MetalFFT.swift:206-277, with fft_transpose and
// fft_twiddle_transpose, Sources/MetalFFT/Resources/fft_multisize.metal:700-749),
// which takes five dispatches and three scalar transposes per transform.
// Here it is two kernels per batch chunk and no separate transpose:
//
//  column pass  x viewed as n1 rows x n2 columns (x[r*n2 + c]).  A CTA takes
//               C = 16 adjacent columns (128-byte row segments; 8 columns
//               when n1 = 1024 to keep the CTA at 512 threads), coalesced,
//               runs the 16 length-n1 FFTs in shared memory, multiplies by
//               W_N^{c*k1} and writes the same positions of a scratch buffer.
//  row pass     A CTA takes 16 consecutive rows k1 of the scratch (one
//               contiguous chunk, read with 16-byte loads into an
//               XOR-swizzled tile), runs the 16 length-n2 FFTs and writes
//               X[k1 + n1*k2] straight to out[k2*n1 + k1]: 16 consecutive k1
//               per k2, i.e. the final transpose is folded into the store.
//
// Output is in natural order, as the reference's last transpose leaves it
// (src/fft_multisize_host.swift:155-164).  Inverse: conjugate on the column
// load, conjugate and scale on the row store (MetalFFT.swift:56-65).
#include "capi_internal.h"
#include "stockham.cuh"

namespace mfft {

constexpr int FS_TILE = 16;  // rows per row-pass CTA (and columns for n1 <= 512)
constexpr int FS_FINE = 1024;
// columns per column-pass CTA: 16 (128-byte row segments), 8 for n1 = 1024 so
// the CTA stays at 512 threads and the line FFT keeps its 16 values in registers
__host__ __device__ constexpr int fs_cols(int L) { return L >= 1024 ? 8 : FS_TILE; }

// W_N^m = fine[m mod 1024] * coarse[m / 1024]; both tables FP64-generated.
__global__ void k_fourstep_tables(float2* fine, float2* coarse, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s, c;
    if (i < FS_FINE) {
        sincospi(-2.0 * (double)i / (double)n, &s, &c);
        fine[i] = make_float2((float)c, (float)s);
    }
    if (i < n / FS_FINE) {
        sincospi(-2.0 * (double)i * FS_FINE / (double)n, &s, &c);
        coarse[i] = make_float2((float)c, (float)s);
    }
}

__device__ __forceinline__ float2 fourstep_twiddle(const float2* __restrict__ fine,
                                                   const float2* __restrict__ coarse, unsigned m) {
    return cmul(__ldg(fine + (m & (FS_FINE - 1))), __ldg(coarse + (m >> 10)));
}

template <int L, bool INV>
__global__ void __launch_bounds__(L / 16 * fs_cols(L)) k_fourstep_cols(const float2* __restrict__ in, float2* __restrict__ out,
                                                     int n2, const float2* __restrict__ tw,
                                                     const float2* __restrict__ fine,
                                                     const float2* __restrict__ coarse) {
    constexpr int E = 16, T = L / E, C = fs_cols(L);
    extern __shared__ float2 smem[];
    const int tiles = n2 / C;
    const long long b = blockIdx.x / tiles;
    const int col = (blockIdx.x % tiles) * C + (threadIdx.x % C);
    const int t = threadIdx.x / C;
    const size_t N = (size_t)L * n2;
    const float2* src = in + b * N + col;
    float2 v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        v[m] = __ldcs(src + (size_t)(t + m * T) * n2);
        if constexpr (INV) v[m].y = -v[m].y;
    }
    fft_regs<L, E, false>(v, t, ColLine<C>{smem, (int)(threadIdx.x % C)}, tw);
    float2* dst = out + b * N + col;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int k1 = t + m * T;
        dst[(size_t)k1 * n2] = cmul(v[m], fourstep_twiddle(fine, coarse, (unsigned)(col * k1)));
    }
}

template <int L, bool INV>
__global__ void __launch_bounds__(L) k_fourstep_rows(const float2* __restrict__ in, float2* __restrict__ out,
                                                     int n1, const float2* __restrict__ tw) {
    constexpr int E = 16, T = L / E, RW = FS_TILE;
    extern __shared__ float2 smem[];
    const int groups = n1 / RW;
    const long long b = blockIdx.x / groups;
    const int row0 = (blockIdx.x % groups) * RW;
    const size_t N = (size_t)n1 * L;
    // RW consecutive rows are one contiguous chunk of RW*L elements.
    const float4* src = reinterpret_cast<const float4*>(in + b * N + (size_t)row0 * L);
    for (int q = threadIdx.x; q < RW * L / 2; q += L) {
        const float4 x = __ldcs(src + q);
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

// ---- host side -------------------------------------------------------------

struct FsKernels {
    int len;
    void (*cols)(const float2*, float2*, int, const float2*, const float2*, const float2*, long long, bool, cudaStream_t);
    void (*rows)(const float2*, float2*, int, const float2*, long long, bool, cudaStream_t);
    cudaError_t (*prepare)();
};

template <int L>
static void launch_cols(const float2* in, float2* out, int n2, const float2* tw, const float2* fine,
                        const float2* coarse, long long nb, bool inv, cudaStream_t s) {
    constexpr int C = fs_cols(L);
    const size_t smem = (size_t)L * C * sizeof(float2);
    const long long blocks = nb * (n2 / C);
    if (inv) k_fourstep_cols<L, true><<<(unsigned)blocks, L / 16 * C, smem, s>>>(in, out, n2, tw, fine, coarse);
    else k_fourstep_cols<L, false><<<(unsigned)blocks, L / 16 * C, smem, s>>>(in, out, n2, tw, fine, coarse);
}

template <int L>
static void launch_rows(const float2* in, float2* out, int n1, const float2* tw, long long nb, bool inv,
                        cudaStream_t s) {
    const size_t smem = (size_t)L * FS_TILE * sizeof(float2);
    const long long blocks = nb * (n1 / FS_TILE);
    if (inv) k_fourstep_rows<L, true><<<(unsigned)blocks, L, smem, s>>>(in, out, n1, tw);
    else k_fourstep_rows<L, false><<<(unsigned)blocks, L, smem, s>>>(in, out, n1, tw);
}

template <int L>
static cudaError_t prepare_fs() {
    const int smem = L * FS_TILE * (int)sizeof(float2);
    const int csmem = L * fs_cols(L) * (int)sizeof(float2);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_fourstep_cols<L, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, csmem))) return e;
    if ((e = cudaFuncSetAttribute(k_fourstep_cols<L, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, csmem))) return e;
    if ((e = cudaFuncSetAttribute(k_fourstep_rows<L, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))) return e;
    return cudaFuncSetAttribute(k_fourstep_rows<L, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

static const FsKernels g_fs[] = {
    {128, &launch_cols<128>, &launch_rows<128>, &prepare_fs<128>},
    {256, &launch_cols<256>, &launch_rows<256>, &prepare_fs<256>},
    {512, &launch_cols<512>, &launch_rows<512>, &prepare_fs<512>},
    {1024, &launch_cols<1024>, &launch_rows<1024>, &prepare_fs<1024>},
};

static const FsKernels* find_fs(int len) {
    for (const auto& k : g_fs)
        if (k.len == len) return &k;
    return nullptr;
}

// n = 2^m, m in [15, 20]: n1 = 2^floor(m/2) (column length), n2 = n / n1.
void fourstep_split(int64_t n, int* n1, int* n2) {
    int m = ilog2c(n);
    *n1 = 1 << (m / 2);
    *n2 = (int)(n / *n1);
}

int fourstep_plan_init(mfft_plan* p) {
    mfft_ctx* ctx = p->ctx;
    FourStep& fs = p->fs;
    fourstep_split(p->n, &fs.n1, &fs.n2);
    const FsKernels* kc = find_fs(fs.n1);
    const FsKernels* kr = find_fs(fs.n2);
    if (!kc || !kr)
        return set_error(MFFT_ERR_KERNEL_NOT_FOUND, -1, -1, -1, "no four-step kernels for %lld", (long long)p->n);
    // twiddle rows of the length-n1 and length-n2 line FFTs (E = 16)
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    const BatchedKernel *bc = nullptr, *br = nullptr;
    for (int i = 0; i < cnt; ++i) {
        if (ks[i].e != 16) continue;
        if (ks[i].n == fs.n1 && !bc) bc = &ks[i];
        if (ks[i].n == fs.n2 && !br) br = &ks[i];
    }
    if (!bc || !br) return set_error(MFFT_ERR_KERNEL_NOT_FOUND, -1, -1, -1, "no line twiddles");
    int st = ctx_twiddles(ctx, bc, &fs.col_tw);
    if (st) return st;
    st = ctx_twiddles(ctx, br, &fs.row_tw);
    if (st) return st;
    cudaError_t e = kc->prepare();
    if (e == cudaSuccess) e = kr->prepare();
    if (e != cudaSuccess) return cuda_error(e, "four-step kernel attributes");
    fs.col = kc;
    fs.row = kr;
    // fine (1024) + coarse (n/1024) twiddle tables
    e = cudaMalloc(&fs.tables, sizeof(float2) * (FS_FINE + p->n / FS_FINE));
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "four-step tables: %s", cudaGetErrorString(e));
    k_fourstep_tables<<<(FS_FINE + 255) / 256, 256, 0, ctx->stream>>>(fs.tables, fs.tables + FS_FINE, (int)p->n);
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(e, "four-step tables");
    // scratch: up to 2^24 complex points per chunk (128 MiB), at least one line
    fs.scratch_lines = (1LL << 24) / p->n;
    if (fs.scratch_lines < 1) fs.scratch_lines = 1;
    e = cudaMalloc(&fs.scratch, sizeof(float2) * (size_t)fs.scratch_lines * (size_t)p->n);
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "four-step scratch: %s", cudaGetErrorString(e));
    return MFFT_SUCCESS;
}

void fourstep_plan_release(mfft_plan* p) {
    if (p->fs.scratch) cudaFree(p->fs.scratch);
    if (p->fs.tables) cudaFree(p->fs.tables);
    p->fs.scratch = nullptr;
    p->fs.tables = nullptr;
}

// Runs the two passes over `batch` lines using `scratch` (room for
// scratch_lines lines) as the intermediate.
int fourstep_run(const FourStep& fs, int64_t n, const float2* in, float2* out, int64_t batch,
                 int direction, float2* scratch, long long scratch_lines, cudaStream_t s) {
    const FsKernels* kc = (const FsKernels*)fs.col;
    const FsKernels* kr = (const FsKernels*)fs.row;
    const bool inv = (direction == MFFT_INVERSE);
    for (int64_t b0 = 0; b0 < batch; b0 += scratch_lines) {
        long long nb = batch - b0 < scratch_lines ? batch - b0 : scratch_lines;
        kc->cols(in + b0 * n, scratch, fs.n2, fs.col_tw, fs.tables, fs.tables + FS_FINE, nb, inv, s);
        kr->rows(scratch, out + b0 * n, fs.n1, fs.row_tw, nb, inv, s);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "four-step launch");
    return MFFT_SUCCESS;
}

int fourstep_exec(mfft_plan* p, const float2* in, float2* out, int64_t batch, int direction, cudaStream_t s) {
    return fourstep_run(p->fs, p->n, in, out, batch, direction, p->fs.scratch, p->fs.scratch_lines, s);
}

}  // namespace mfft

extern "C" int mfft_plan_set_fourstep_chunk(mfft_plan* plan, int64_t lines) {
    using namespace mfft;
    if (!plan) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    if (plan->n <= MFFT_MAX_SINGLE_N)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "n=%lld has no four-step chunk", (long long)plan->n);
    if (lines < 1) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, lines, -1, "lines must be >= 1");
    DeviceGuard g(plan->ctx->device);
    FourStep& fs = plan->fs;
    if (lines > fs.scratch_lines) {
        float2* s = nullptr;
        cudaError_t e = cudaMalloc(&s, sizeof(float2) * (size_t)lines * (size_t)plan->n);
        if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "four-step scratch: %s", cudaGetErrorString(e));
        cudaFree(fs.scratch);
        fs.scratch = s;
    }
    fs.scratch_lines = lines;
    return MFFT_SUCCESS;
}
