// capi_internal.h -- handle layouts and helpers shared by the C-ABI sources.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <functional>
#include <map>
#include <mutex>
#include <utility>

#include "../../include/mfft.h"
#include "kernels.h"

namespace mfft {
struct HostCopier;
void host_copier_free(HostCopier* c);
}  // namespace mfft

#define MFFT_MAX_N (1 << 20)
#define MFFT_MAX_SINGLE_N 16384

struct mfft_ctx {
    int device = 0;
    int sms = 0;
    int l2_bytes = 0;
    bool shared = false;
    cudaStream_t stream = nullptr;
    int* dev_err = nullptr;   // device word: first bounded-wait failure of any kernel
    std::mutex mu;
    std::map<std::pair<int, int>, float2*> twiddles;     // (n, e) -> twiddle rows
    std::map<int, const mfft::BatchedKernel*> tuned;     // n -> autotuned kernel
    std::map<int, int> tuned_split;                      // log2 n -> autotuned log2 n1 (four-step)
    // host-array calls: a memory pool that keeps its memory between calls,
    // and the chunked pipeline of line-independent transforms (upload and
    // download streams, staging slots, one event ring per stage)
    cudaMemPool_t pool = nullptr;
    std::mutex stage_mu;
    cudaStream_t h2d = nullptr, d2h = nullptr;
    void* stage = nullptr;
    cudaEvent_t ev_up[4] = {}, ev_done[4] = {}, ev_down[4] = {};
    // pageable host arrays: pinned host slots (in and out per staging slot)
    // filled and drained by a small pool of host threads
    void* hstage = nullptr;
    mfft::HostCopier* copier = nullptr;
};

namespace mfft {

struct BatchedBinding {
    const BatchedKernel* k = nullptr;
    float2* tw = nullptr;
};

// Four-step state for n > 16384 (n = n1 * n2, n1 <= n2 <= 1024), run by the
// item kernel of fsqueue.cu.
struct FourStep {
    int n1 = 0, n2 = 0;
    int l1 = 0;                  // log2 n1
    float2* col_tw = nullptr;    // line twiddle rows for n1 and n2
    float2* row_tw = nullptr;
    float2* tables = nullptr;    // W_N^m = fine[m % 1024] * coarse[m / 1024]
    float2* scratch = nullptr;   // intermediates of up to scratch_lines transforms
    long long scratch_lines = 0;
};

struct TcState {
    void* dft_tables = nullptr;  // device: realified DFT16 operands (hi/lo, bf16)
    float2* tw = nullptr;        // device: inter-stage twiddles
    bool ready = false;
};

}  // namespace mfft

struct mfft_plan {
    mfft_ctx* ctx = nullptr;
    int64_t n = 0;
    mfft::BatchedBinding line;
    mfft::FourStep fs;
    mfft::TcState tc;
};

namespace mfft {

int set_error(int status, int64_t expected, int64_t got, int64_t index, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what);
bool is_pow2_in(int64_t n, int64_t lo, int64_t hi);

struct DeviceGuard {
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
    int prev_ = 0;
};

int ctx_twiddles(mfft_ctx* ctx, const BatchedKernel* k, float2** out);
int bind_batched(mfft_ctx* ctx, const BatchedKernel* k, BatchedBinding* b);
const BatchedKernel* tuned_batched(mfft_ctx* ctx, int n);

int check_exec_args(const void* in, void* out, int64_t batch, int direction, int flags);
// adjoint = 1: the adjoint (conjugate transpose) of the transform in
// `direction` instead of the transform (mfft_exec_c2c_backward)
int launch_c2c_device(mfft_plan* plan, const float2* in, float2* out, int64_t batch, int direction,
                      cudaStream_t s, int adjoint = 0);
int check_device_error(mfft_ctx* ctx);
// Host-array call: copy in, run `body` on device buffers, copy out, wait.
// in_place: the kernels may read and write one buffer (batched FFTs).
// Host arrays of `lines` independent lines (in_line / out_line bytes each):
// chunks of <= STAGE_SLOT_BYTES are uploaded on ctx->h2d, transformed in order
// on ctx->stream by body(d_in, d_out, chunk_lines, stream) and downloaded on
// ctx->d2h, so that the two copy directions and the transforms overlap;
// `pair` keeps chunk boundaries on even lines.  Returns after the last
// download.  Falls back to run_host_staged for one chunk.
constexpr size_t STAGE_SLOT_BYTES = 16u << 20;
constexpr int STAGE_SLOTS = 4;
int run_host_lines(mfft_ctx* ctx, const void* in, void* out, int64_t lines, size_t in_line, size_t out_line,
                   const std::function<int(const void* d_in, void* d_out, int64_t lines, cudaStream_t)>& body,
                   bool in_place, bool pair = false);
int run_host_staged(mfft_ctx* ctx, const void* in, void* out, size_t in_bytes, size_t out_bytes,
                    const std::function<int(void* d_in, void* d_out, cudaStream_t)>& body, bool in_place = false);

// FusedConvolver FP16 forward kernels (fft 4096, conv_fp16.cu): resident
// CTAs per SM of a mode (0 if its attributes cannot be set), and the launch
// with the FP32 forward kernel's walker arguments.
int conv_fp16_ctas_per_sm(int mode);
cudaError_t conv_fp16_forward(int mode, long long ctas, cudaStream_t s, const float* x, long long nx, float* y,
                              long long ny, const float2* H, const float2* tw, int hop, long long npairs,
                              long long ppu, int warm);

// Line twiddle rows (E = 16) of size n, cached in the context.
int line_twiddles(mfft_ctx* ctx, int n, float2** out);
// W_n^m tables (fine[1024] then coarse[n / 1024]) for a four-step size n,
// built on the context's stream; the caller owns the allocation.
int fourstep_tables(mfft_ctx* ctx, int64_t n, float2** out);

// Four-step sizes whose tiles move by TMA (2^16 .. 2^20), and one pass
// (FSQ_COLS or FSQ_ROWS) of them over nb contiguous transforms of 2^logn
// points: in / out / scratch are the first transform's data (fsqueue.h).
// Tensor map of `rows` rows of `row_points` complex values at `base`, boxes of
// tile_cols complex columns x box_rows rows with the item tiles' swizzle (32,
// 64 or 128 bytes for 4, 8 or 16 columns).
bool encode_rows(CUtensorMap* map, const float2* base, uint64_t rows, uint64_t row_points, int tile_cols,
                 int box_rows = 256);
struct FsqTables;
int fourstep_tma_pass(int kind, const FsqTables& tabs, const float2* in, float2* out, float2* scratch, long long nb,
                      int logn, int l1, bool inv, mfft_ctx* ctx, cudaStream_t s, int adjoint = 0);

int fourstep_plan_init(mfft_plan* plan);
// (Re)binds a four-step plan to the split n1 = 2^l1 (twiddle rows of n1 and n2).
int fourstep_set_split(mfft_plan* plan, int l1);
// The split a new four-step plan of 2^logn points takes in this context: the
// autotuned one, else one read from $MFFT_TUNE_CACHE, else the default.
int fourstep_split_for(mfft_ctx* ctx, int logn);
void fourstep_plan_release(mfft_plan* plan);
int fourstep_exec(mfft_plan* plan, const float2* in, float2* out, int64_t batch, int direction,
                  cudaStream_t s, int adjoint = 0);

int tc_plan_init(mfft_plan* plan);
void tc_plan_release(mfft_plan* plan);

}  // namespace mfft
