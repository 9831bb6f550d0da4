// autotune.cu -- per-size choice of the batched kernel (radix E, lines per
// CTA) by timing the candidates on the device, cached per context and on disk.
//
// The reference fixes one kernel and thread count per size in a switch
// (FFTDescriptor, Sources/MetalFFT/Internal/MetalContext.swift:47-69; N=4096
// batches switch to the radix-8 kernel, MetalFFT.swift:163-165).  Here every
// registered instantiation for the size is timed with CUDA events on a batch
// larger than L2 and the fastest is kept.  The cache file (one line
// "n e fpb stages" per size) is read from $MFFT_TUNE_CACHE when that is set.
//
// Sizes above 16384 run the four-step FFT n = n1 x n2; the reference fixes
// n1 = 2^floor(log2(n)/2) (FourStepFFT.swift).  mfft_autotune_fourstep times
// every admissible split (64 <= n1 <= 1024, 128 <= n2 <= 1024) and keeps the
// fastest.
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "capi_internal.h"
#include "fft_common.cuh"
#include "fsqueue.h"

namespace mfft {

static bool read_cache(int n, int* e, int* fpb, int* st) {
    const char* path = getenv("MFFT_TUNE_CACHE");
    if (!path || !*path) return false;
    FILE* f = fopen(path, "r");
    if (!f) return false;
    int cn, ce, cf, cs;
    bool found = false;
    while (fscanf(f, "%d %d %d %d", &cn, &ce, &cf, &cs) == 4) {
        if (cn == n) {
            *e = ce;
            *fpb = cf;
            *st = cs;
            found = true;
        }
    }
    fclose(f);
    return found;
}

static void write_cache(int n, int e, int fpb, int st) {
    const char* path = getenv("MFFT_TUNE_CACHE");
    if (!path || !*path) return;
    FILE* f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "%d %d %d %d\n", n, e, fpb, st);
    fclose(f);
}

const BatchedKernel* tuned_batched(mfft_ctx* ctx, int n) {
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->tuned.find(n);
        if (it != ctx->tuned.end()) return it->second;
    }
    const BatchedKernel* k = nullptr;
    int e = 0, fpb = 0, st = 0;
    if (read_cache(n, &e, &fpb, &st)) k = find_batched(n, e, fpb, st);
    if (!k) k = default_batched(n);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->tuned[n] = k;
    return k;
}

// Times every registered candidate for size n on `lines` lines and installs
// the fastest in the context.  Returns the chosen kernel through out.
int autotune_batched(mfft_ctx* ctx, int n, long long lines, const BatchedKernel** out) {
    DeviceGuard g(ctx->device);
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    size_t bytes = (size_t)lines * n * sizeof(float2);
    float2 *a = nullptr, *b = nullptr;
    if (cudaMalloc(&a, bytes) != cudaSuccess || cudaMalloc(&b, bytes) != cudaSuccess) {
        cudaFree(a);
        return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "autotune buffers");
    }
    cudaMemsetAsync(a, 0, bytes, ctx->stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const BatchedKernel* best = nullptr;
    float best_ms = 1e30f;
    for (int i = 0; i < cnt; ++i) {
        if (ks[i].n != n) continue;
        BatchedBinding bb;
        if (bind_batched(ctx, &ks[i], &bb) != MFFT_SUCCESS) continue;
        for (int w = 0; w < 3; ++w) ks[i].fwd(a, b, lines, bb.tw, ctx->dev_err, ctx->stream, 0);
        cudaEventRecord(e0, ctx->stream);
        const int reps = 10;
        for (int r = 0; r < reps; ++r)
            ks[i].fwd((r & 1) ? b : a, (r & 1) ? a : b, lines, bb.tw, ctx->dev_err, ctx->stream, 0);
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) continue;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
            best_ms = ms;
            best = &ks[i];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(a);
    cudaFree(b);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_error(err, "autotune");
    if (!best) return set_error(MFFT_ERR_KERNEL_NOT_FOUND, -1, -1, -1, "no kernel for n=%d", n);
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->tuned[n] = best;
    }
    write_cache(n, best->e, best->fpb, best->stages);
    *out = best;
    return MFFT_SUCCESS;
}

// Four-step splits share the cache file: a line "n n1 0 0" with n > 16384
// records the split n = n1 x n/n1 chosen for that size.
int fourstep_split_for(mfft_ctx* ctx, int logn) {
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->tuned_split.find(logn);
        if (it != ctx->tuned_split.end()) return it->second;
    }
    int l1 = fsq_default_l1(logn);
    int n1 = 0, z0 = 0, z1 = 0;
    if (read_cache(1 << logn, &n1, &z0, &z1) && n1 > 0 && (n1 & (n1 - 1)) == 0 && fsq_split_ok(logn, ilog2c(n1)))
        l1 = ilog2c(n1);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->tuned_split[logn] = l1;
    return l1;
}

// Times the plan's four-step FFT for every admissible split over `batch`
// transforms and leaves the plan on the fastest; the choice is installed in
// the context for later plans of the size and appended to the cache file.
static int autotune_split(mfft_plan* p, long long batch, int* out_l1) {
    mfft_ctx* ctx = p->ctx;
    const int logn = ilog2c(p->n);
    const size_t bytes = (size_t)batch * (size_t)p->n * sizeof(float2);
    float2 *a = nullptr, *b = nullptr;
    if (cudaMalloc(&a, bytes) != cudaSuccess || cudaMalloc(&b, bytes) != cudaSuccess) {
        cudaFree(a);
        return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "autotune buffers");
    }
    cudaMemsetAsync(a, 0, bytes, ctx->stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int l1_was = p->fs.l1;
    int best = -1, st = MFFT_SUCCESS;
    float best_ms = 1e30f;
    for (int l1 = 6; l1 <= 10 && !st; ++l1) {
        if (!fsq_split_ok(logn, l1)) continue;
        st = fourstep_set_split(p, l1);
        for (int w = 0; w < 2 && !st; ++w) st = fourstep_exec(p, a, b, batch, MFFT_FORWARD, ctx->stream, 0);
        if (st) break;
        cudaEventRecord(e0, ctx->stream);
        const int reps = 6;
        for (int r = 0; r < reps && !st; ++r)
            st = fourstep_exec(p, (r & 1) ? b : a, (r & 1) ? a : b, batch, MFFT_FORWARD, ctx->stream, 0);
        cudaEventRecord(e1, ctx->stream);
        if (st) break;
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            st = cuda_error(e, "four-step autotune");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
            best_ms = ms;
            best = l1;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(a);
    cudaFree(b);
    if (st || best < 0) {
        fourstep_set_split(p, l1_was);
        return st ? st : set_error(MFFT_ERR_KERNEL_NOT_FOUND, -1, -1, -1, "no four-step split for n=%lld",
                                   (long long)p->n);
    }
    st = fourstep_set_split(p, best);
    if (st) return st;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->tuned_split[logn] = best;
    }
    write_cache((int)p->n, 1 << best, 0, 0);
    *out_l1 = best;
    return MFFT_SUCCESS;
}

}  // namespace mfft

extern "C" int mfft_autotune_fourstep(mfft_plan* plan, int64_t batch, int* n1) {
    using namespace mfft;
    if (!plan) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    if (plan->n <= MFFT_MAX_SINGLE_N)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "n=%lld does not use the four-step path",
                         (long long)plan->n);
    if (batch <= 0) batch = std::max<int64_t>(1, (int64_t)(512ll << 20) / (plan->n * 8));  // 512 MiB, 4x L2
    DeviceGuard g(plan->ctx->device);
    int l1 = 0;
    int st = autotune_split(plan, batch, &l1);
    if (st) return st;
    if (n1) *n1 = 1 << l1;
    return check_device_error(plan->ctx);
}

extern "C" int mfft_plan_set_split(mfft_plan* plan, int64_t n1) {
    using namespace mfft;
    if (!plan) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    if (plan->n <= MFFT_MAX_SINGLE_N)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "n=%lld does not use the four-step path",
                         (long long)plan->n);
    if (n1 <= 0 || (n1 & (n1 - 1)))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, n1, -1, "n1 = %lld is not a power of two", (long long)n1);
    DeviceGuard g(plan->ctx->device);
    return fourstep_set_split(plan, ilog2c(n1));
}

extern "C" int mfft_plan_split(const mfft_plan* plan, int64_t* n1, int64_t* n2) {
    if (!plan) return mfft::set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    const bool fs = plan->n > MFFT_MAX_SINGLE_N;
    if (n1) *n1 = fs ? plan->fs.n1 : 0;
    if (n2) *n2 = fs ? plan->fs.n2 : 0;
    return MFFT_SUCCESS;
}

extern "C" int mfft_list_splits(int64_t n, int64_t* n1, int cap) {
    int m = 0;
    if (n <= MFFT_MAX_SINGLE_N || n > MFFT_MAX_N || (n & (n - 1))) return 0;
    const int logn = mfft::ilog2c(n);
    for (int l1 = 6; l1 <= 10; ++l1) {
        if (!mfft::fsq_split_ok(logn, l1)) continue;
        if (m < cap && n1) n1[m] = 1LL << l1;
        ++m;
    }
    return m;
}

extern "C" int mfft_autotune(mfft_ctx* ctx, int64_t n, int64_t lines, int* radix, int* lines_per_cta,
                             int* stages) {
    using namespace mfft;
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    if (!is_pow2_in(n, 64, MFFT_MAX_SINGLE_N))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, n, -1, -1, "autotune covers 64..16384, got %lld", (long long)n);
    if (lines <= 0) lines = (int64_t)(256ll << 20) / (n * 8);  // 256 MiB, twice L2
    const BatchedKernel* k = nullptr;
    int st = autotune_batched(ctx, (int)n, lines, &k);
    if (st) return st;
    if (radix) *radix = k->e;
    if (lines_per_cta) *lines_per_cta = k->fpb;
    if (stages) *stages = k->stages;
    return check_device_error(ctx);
}

extern "C" int mfft_plan_kernel_info(const mfft_plan* plan, int* radix, int* lines_per_cta, int* threads,
                                     int* stages) {
    if (!plan) return mfft::set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    const mfft::BatchedKernel* k = plan->line.k;
    if (radix) *radix = k ? k->e : 16;
    if (lines_per_cta) *lines_per_cta = k ? k->fpb : 0;
    if (threads) *threads = k ? k->threads : 0;
    if (stages) *stages = k ? k->stages : 0;
    return MFFT_SUCCESS;
}

extern "C" int mfft_plan_set_kernel(mfft_plan* plan, int radix, int lines_per_cta, int stages) {
    using namespace mfft;
    if (!plan) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    if (plan->n > MFFT_MAX_SINGLE_N)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "n=%lld uses the four-step path", (long long)plan->n);
    const BatchedKernel* k = find_batched((int)plan->n, radix, lines_per_cta, stages);
    if (!k)
        return set_error(MFFT_ERR_KERNEL_NOT_FOUND, -1, -1, -1,
                         "no variant n=%lld radix=%d lines_per_cta=%d stages=%d", (long long)plan->n, radix,
                         lines_per_cta, stages);
    DeviceGuard g(plan->ctx->device);
    return bind_batched(plan->ctx, k, &plan->line);
}

extern "C" int mfft_list_kernels(int64_t n, int* radix, int* lines_per_cta, int* stages, int cap) {
    int cnt = 0, m = 0;
    const mfft::BatchedKernel* ks = mfft::batched_kernels(&cnt);
    for (int i = 0; i < cnt; ++i) {
        if (ks[i].n != n) continue;
        if (m < cap) {
            if (radix) radix[m] = ks[i].e;
            if (lines_per_cta) lines_per_cta[m] = ks[i].fpb;
            if (stages) stages[m] = ks[i].stages;
        }
        ++m;
    }
    return m;
}
