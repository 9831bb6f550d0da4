// fourstep.cu -- C2C FFT for N = 2^15 .. 2^20 as N = n1 * n2 (n1 <= n2 <= 1024).
//
// B200 form of the reference's four-step plan (dispatchFourStep,
// Sources/MetalFFT/FFT/MetalFFT.swift:206-277, with fft_transpose and
// fft_twiddle_transpose, Sources/MetalFFT/Resources/fft_multisize.metal:700-749),
// which takes five dispatches and three scalar transposes per transform and
// one command buffer per batch element.  Here a batch (up to 2^25 points at a
// time) is two launches of the item kernel (fsqueue.cu) and no transpose pass
// exists:
//
//  column pass   x viewed as n1 rows x n2 columns (x[r*n2 + c]).  An item is
//                4096/n1 adjacent columns (16-byte chunks of every row),
//                whose n1-point FFTs are multiplied by W_N^{c*k1} and stored
//                at the same positions of a scratch area;
//  row pass      4096/n2 consecutive rows k1 of the scratch (one contiguous
//                chunk); their n2-point FFTs give X[k1 + n1*k2], stored
//                straight to out[k2*n1 + k1] through a shared-memory tile,
//                i.e. the final transpose is folded into the store.
//
// Output is in natural order, as the reference's last transpose leaves it
// (src/fft_multisize_host.swift:155-164).  Inverse: conjugate on the column
// load, conjugate and scale on the row store (MetalFFT.swift:56-65).
#include <cudaTypedefs.h>

#include <mutex>

#include "capi_internal.h"
#include "fsqueue.h"
#include "stockham.cuh"

namespace mfft {

constexpr int FS_FINE = 1024;

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

int line_twiddles(mfft_ctx* ctx, int n, float2** out) {
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    for (int i = 0; i < cnt; ++i)
        if (ks[i].n == n && ks[i].e == 16) return ctx_twiddles(ctx, &ks[i], out);
    return set_error(MFFT_ERR_KERNEL_NOT_FOUND, -1, -1, -1, "no line twiddles for n=%d", n);
}

int fourstep_tables(mfft_ctx* ctx, int64_t n, float2** out) {
    *out = nullptr;
    float2* t = nullptr;
    cudaError_t e = cudaMalloc(&t, sizeof(float2) * (size_t)(FS_FINE + n / FS_FINE));
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "four-step tables: %s", cudaGetErrorString(e));
    k_fourstep_tables<<<(FS_FINE + 255) / 256, 256, 0, ctx->stream>>>(t, t + FS_FINE, (int)n);
    e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFree(t);
        return cuda_error(e, "four-step tables");
    }
    *out = t;
    return MFFT_SUCCESS;
}

int fourstep_set_split(mfft_plan* p, int l1) {
    FourStep& fs = p->fs;
    const int logn = ilog2c(p->n);
    if (!fsq_split_ok(logn, l1))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, 1LL << l1, -1,
                         "n1 = %d is not a valid four-step split of n = %lld (64 <= n1 <= 1024, 128 <= n/n1 <= 1024)",
                         1 << l1, (long long)p->n);
    int n1, n2;
    fsq_split(logn, &n1, &n2, l1);
    float2 *ct = nullptr, *rt = nullptr;
    int st = line_twiddles(p->ctx, n1, &ct);
    if (!st) st = line_twiddles(p->ctx, n2, &rt);
    if (st) return st;
    fs.l1 = l1;
    fs.n1 = n1;
    fs.n2 = n2;
    fs.col_tw = ct;
    fs.row_tw = rt;
    return MFFT_SUCCESS;
}

int fourstep_plan_init(mfft_plan* p) {
    mfft_ctx* ctx = p->ctx;
    FourStep& fs = p->fs;
    const int logn = ilog2c(p->n);
    int st = fourstep_set_split(p, fourstep_split_for(ctx, logn));
    if (!st) st = fourstep_tables(ctx, p->n, &fs.tables);
    if (st) return st;
    cudaError_t e = fsq_prepare();
    if (e != cudaSuccess) return cuda_error(e, "four-step kernel attributes");
    // intermediates of up to 2^25 points (256 MiB) per pair of passes
    fs.scratch_lines = (1LL << 25) / p->n;
    e = cudaMalloc(&fs.scratch, sizeof(float2) * (size_t)fs.scratch_lines * (size_t)p->n);
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "four-step scratch: %s", cudaGetErrorString(e));
    return MFFT_SUCCESS;
}

void fourstep_plan_release(mfft_plan* p) {
    cudaFree(p->fs.scratch);
    cudaFree(p->fs.tables);
    p->fs.scratch = nullptr;
    p->fs.tables = nullptr;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

// `rows` rows of `row_points` complex values at `base`, as floats; boxes of
// `tile_cols` complex columns x box_rows rows, swizzled like the item tiles
bool encode_rows(CUtensorMap* map, const float2* base, uint64_t rows, uint64_t row_points, int tile_cols,
                 int box_rows) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {2 * row_points, rows};
    const cuuint64_t strides[1] = {row_points * sizeof(float2)};
    const cuuint32_t box[2] = {(cuuint32_t)(2 * tile_cols), (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUtensorMapSwizzle sw = tile_cols == 4   ? CU_TENSOR_MAP_SWIZZLE_32B
                                  : tile_cols == 8 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                   : CU_TENSOR_MAP_SWIZZLE_128B;
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float2*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}


int fourstep_tma_pass(int kind, const FsqTables& tabs, const float2* in, float2* out, float2* scratch, long long nb,
                      int logn, int l1, bool inv, mfft_ctx* ctx, cudaStream_t s, int adjoint) {
    int n1, n2;
    fsq_split(logn, &n1, &n2, l1);
    FsqArgs a{};
    a.in = in;
    a.out = out;
    a.scratch = scratch;
    a.u_logn = logn;
    a.u_l1 = l1;
    a.adjoint = adjoint;
    a.tabs = tabs;
    FsqMaps m{};
    bool ok;
    if (kind == FSQ_COLS) {
        const int C = FSQ_POINTS / n1;
        ok = encode_rows(&m.ld, in, (uint64_t)nb * n1, n2, C) && encode_rows(&m.st, scratch, (uint64_t)nb * n1, n2, C);
        a.u_per = fsq_cols_items(logn);
    } else {
        ok = encode_rows(&m.st, out, (uint64_t)nb * n2, n1, FSQ_POINTS / n2);
        a.u_per = fsq_rows_items(logn);
    }
    if (!ok) return set_error(MFFT_ERR_LIBRARY_BUILD, -1, -1, -1, "four-step tensor maps could not be encoded");
    a.u_kind = kind;
    a.nitems = (int)(nb * a.u_per);
    cudaError_t e = fsq_launch_tma(a, m, inv, ctx->sms, ctx->dev_err, s);
    return e == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(e, "four-step launch");
}

// Column pass then row pass over chunks of up to scratch_lines transforms;
// splits with n1, n2 in {256, 512, 1024} move their tiles with TMA (tile
// widths 16, 8 or 4), the others with 16-byte copies.
int fourstep_exec(mfft_plan* p, const float2* in, float2* out, int64_t batch, int direction, cudaStream_t s,
                  int adjoint) {
    const FourStep& fs = p->fs;
    const int logn = ilog2c(p->n);
    const int nc = fsq_cols_items(logn), nr = fsq_rows_items(logn);
    FsqArgs a{};
    a.scratch = fs.scratch;
    a.u_logn = logn;
    a.u_l1 = fs.l1;
    a.adjoint = adjoint;
    a.tabs.line_tw[ilog2c(fs.n1) - 6] = fs.col_tw;
    a.tabs.line_tw[ilog2c(fs.n2) - 6] = fs.row_tw;
    a.tabs.fine[logn - 13] = fs.tables;
    a.tabs.coarse[logn - 13] = fs.tables + FS_FINE;
    const bool inv = direction == MFFT_INVERSE;
    for (int64_t b0 = 0; b0 < batch; b0 += fs.scratch_lines) {
        const long long nb = batch - b0 < fs.scratch_lines ? batch - b0 : fs.scratch_lines;
        a.in = in + b0 * p->n;
        a.out = out + b0 * p->n;
        if (fsq_tma_split(logn, fs.l1)) {
            int st = fourstep_tma_pass(FSQ_COLS, a.tabs, a.in, a.out, a.scratch, nb, logn, fs.l1, inv, p->ctx, s,
                                       adjoint);
            if (!st)
                st = fourstep_tma_pass(FSQ_ROWS, a.tabs, a.in, a.out, a.scratch, nb, logn, fs.l1, inv, p->ctx, s,
                                       adjoint);
            if (st) return st;
            continue;
        }
        a.u_kind = FSQ_COLS;
        a.u_per = nc;
        a.nitems = (int)(nb * nc);
        cudaError_t e = fsq_launch(a, inv, p->ctx->sms, s);
        if (e == cudaSuccess) {
            a.u_kind = FSQ_ROWS;
            a.u_per = nr;
            a.nitems = (int)(nb * nr);
            e = fsq_launch(a, inv, p->ctx->sms, s);
        }
        if (e != cudaSuccess) return cuda_error(e, "four-step launch");
    }
    return MFFT_SUCCESS;
}

}  // namespace mfft
