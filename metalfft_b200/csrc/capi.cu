// capi.cu -- the extern "C" boundary of libmfft (include/mfft.h): contexts,
// plans, error reporting and the batched C2C entry points.
//
// Mirrors the reference runtime (Sources/MetalFFT/Internal/MetalContext.swift,
// Dispatch.swift, Sources/MetalFFT/FFT/MetalFFT.swift): a lock-protected
// process-wide context per device (MetalContext.shared, :74-88), a plan per
// size (FFTDescriptor, :34-70), synchronous host-array calls that surface a
// failed execution as MFFT_ERR_EXEC_FAILED (commitAndWait, Dispatch.swift:3-10).
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <condition_variable>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "capi_internal.h"
#include "tma.cuh"

using namespace mfft;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

namespace {
struct ErrState {
    int status = MFFT_SUCCESS;
    std::string msg;
    int64_t expected = -1, got = -1, index = -1;
};
thread_local ErrState g_err;
}  // namespace

namespace mfft {

int set_error(int status, int64_t expected, int64_t got, int64_t index, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err.status = status;
    g_err.msg = buf;
    g_err.expected = expected;
    g_err.got = got;
    g_err.index = index;
    return status;
}

int cuda_error(cudaError_t e, const char* what) {
    return set_error(e == cudaErrorMemoryAllocation ? MFFT_ERR_ALLOCATION : MFFT_ERR_EXEC_FAILED, -1,
                     -1, -1, "Command buffer error: %s: %s", what, cudaGetErrorString(e));
}

DeviceGuard::DeviceGuard(int dev) {
    cudaGetDevice(&prev_);
    if (prev_ != dev) cudaSetDevice(dev);
}
DeviceGuard::~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != prev_) cudaSetDevice(prev_);
}

bool is_pow2_in(int64_t n, int64_t lo, int64_t hi) {
    return n >= lo && n <= hi && (n & (n - 1)) == 0;
}

}  // namespace mfft

extern "C" const char* mfft_status_string(int status) {
    switch (status) {
        case MFFT_SUCCESS: return "success";
        case MFFT_ERR_NO_DEVICE: return "No CUDA device available";
        case MFFT_ERR_NO_STREAM: return "Could not create CUDA stream";
        case MFFT_ERR_LIBRARY_BUILD: return "Kernel image not loadable on this device (needs sm_100a)";
        case MFFT_ERR_KERNEL_NOT_FOUND: return "Kernel not found";
        case MFFT_ERR_EXEC_FAILED: return "Command buffer error";
        case MFFT_ERR_INVALID_INPUT_SIZE: return "Input size mismatch";
        case MFFT_ERR_BATCH_INPUT_SIZE: return "Batch element size mismatch";
        case MFFT_ERR_UNSUPPORTED_SIZE: return "Unsupported FFT size";
        case MFFT_ERR_ALLOCATION: return "Device buffer allocation failed";
        case MFFT_ERR_INVALID_ARGUMENT: return "Invalid argument";
        case MFFT_ERR_TIMEOUT: return "Device-side wait timed out";
        default: return "unknown status";
    }
}

extern "C" int mfft_last_error(char* buf, size_t len) {
    if (buf && len) {
        size_t n = g_err.msg.size() < len - 1 ? g_err.msg.size() : len - 1;
        memcpy(buf, g_err.msg.data(), n);
        buf[n] = 0;
    }
    return g_err.status;
}

extern "C" int mfft_last_error_detail(int64_t* expected, int64_t* got, int64_t* index) {
    if (expected) *expected = g_err.expected;
    if (got) *got = g_err.got;
    if (index) *index = g_err.index;
    return g_err.status;
}

// ---------------------------------------------------------------------------
// contexts
// ---------------------------------------------------------------------------

static int ctx_init(int device, mfft_ctx** out) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "No CUDA device available (%s)",
                         cudaGetErrorString(e));
    if (device < 0) {
        if (cudaGetDevice(&device) != cudaSuccess) device = 0;
    }
    if (device >= count)
        return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "CUDA device %d does not exist (%d present)",
                         device, count);
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "%s", cudaGetErrorString(e));
    if (prop.major != 10 || prop.minor != 0)
        return set_error(MFFT_ERR_LIBRARY_BUILD, -1, -1, -1,
                         "libmfft is built for sm_100a only; device %d is sm_%d%d (%s)", device,
                         prop.major, prop.minor, prop.name);
    DeviceGuard g(device);
    mfft_ctx* c = new mfft_ctx();
    c->device = device;
    c->sms = prop.multiProcessorCount;
    c->l2_bytes = prop.l2CacheSize;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return set_error(MFFT_ERR_NO_STREAM, -1, -1, -1, "Could not create CUDA stream: %s",
                         cudaGetErrorString(e));
    }
    e = cudaMalloc(&c->dev_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->dev_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "context error word: %s", cudaGetErrorString(e));
    }
    *out = c;
    return MFFT_SUCCESS;
}

static std::mutex g_shared_mu;
static mfft_ctx* g_shared[64];

extern "C" int mfft_context_shared(mfft_ctx** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    int dev = 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "No CUDA device available");
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(MFFT_ERR_NO_DEVICE, -1, -1, -1, "device %d", dev);
    std::lock_guard<std::mutex> lk(g_shared_mu);
    if (!g_shared[dev]) {
        mfft_ctx* c = nullptr;
        int st = ctx_init(dev, &c);
        if (st) return st;
        c->shared = true;
        g_shared[dev] = c;
    }
    *out = g_shared[dev];
    return MFFT_SUCCESS;
}

extern "C" int mfft_context_create(int device, mfft_ctx** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    return ctx_init(device, out);
}

extern "C" int mfft_context_destroy(mfft_ctx* ctx) {
    if (!ctx) return MFFT_SUCCESS;
    if (ctx->shared)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "the shared context is never destroyed");
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->h2d) {
        cudaStreamSynchronize(ctx->h2d);
        cudaStreamSynchronize(ctx->d2h);
        cudaStreamDestroy(ctx->h2d);
        cudaStreamDestroy(ctx->d2h);
        for (int i = 0; i < mfft::STAGE_SLOTS; ++i) {
            cudaEventDestroy(ctx->ev_up[i]);
            cudaEventDestroy(ctx->ev_done[i]);
            cudaEventDestroy(ctx->ev_down[i]);
        }
        cudaFree(ctx->stage);
    }
    if (ctx->hstage) cudaFreeHost(ctx->hstage);
    mfft::host_copier_free(ctx->copier);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    for (auto& kv : ctx->twiddles) cudaFree(kv.second);
    cudaFree(ctx->dev_err);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MFFT_SUCCESS;
}

extern "C" int mfft_context_sm_count(const mfft_ctx* ctx) { return ctx ? ctx->sms : 0; }

extern "C" int mfft_context_check(mfft_ctx* ctx) {
    if (!ctx) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "ctx is NULL");
    DeviceGuard g(ctx->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_error(e, "execution");
    return check_device_error(ctx);
}

namespace mfft {

// Twiddle rows of a (kernel n, e) pair, built once per context on the device.
int ctx_twiddles(mfft_ctx* ctx, const BatchedKernel* k, float2** out) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto key = std::make_pair(k->n, k->e);
    auto it = ctx->twiddles.find(key);
    if (it != ctx->twiddles.end()) {
        *out = it->second;
        return MFFT_SUCCESS;
    }
    float2* tw = nullptr;
    cudaError_t e = cudaMalloc(&tw, sizeof(float2) * (size_t)k->tw_size);
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "twiddle table: %s", cudaGetErrorString(e));
    k->gen_twiddles(tw, ctx->stream);
    e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFree(tw);
        return cuda_error(e, "twiddle generation");
    }
    ctx->twiddles[key] = tw;
    *out = tw;
    return MFFT_SUCCESS;
}

int bind_batched(mfft_ctx* ctx, const BatchedKernel* k, BatchedBinding* b) {
    cudaError_t e = k->prepare();
    if (e != cudaSuccess) return cuda_error(e, "kernel attributes");
    b->k = k;
    return ctx_twiddles(ctx, k, &b->tw);
}

}  // namespace mfft

// ---------------------------------------------------------------------------
// plans
// ---------------------------------------------------------------------------

extern "C" int64_t mfft_recommended_fft_size(int64_t kernel_count) {
    static const int64_t sizes[] = {64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384};
    for (int64_t s : sizes)
        if (s > kernel_count) return s;
    return 0;
}

extern "C" int mfft_plan_create(mfft_ctx* ctx, int64_t n, mfft_plan** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    *out = nullptr;
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    if (!is_pow2_in(n, 64, MFFT_MAX_N))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, n, -1, -1,
                         "Unsupported FFT size: %lld. Supported: powers of two 64..%d", (long long)n,
                         MFFT_MAX_N);
    DeviceGuard g(ctx->device);
    mfft_plan* p = new mfft_plan();
    p->ctx = ctx;
    p->n = n;
    int st = MFFT_SUCCESS;
    if (n <= MFFT_MAX_SINGLE_N) {
        const BatchedKernel* k = tuned_batched(ctx, (int)n);
        if (!k) {
            delete p;
            return set_error(MFFT_ERR_KERNEL_NOT_FOUND, -1, -1, -1, "no batched kernel for n=%lld", (long long)n);
        }
        st = bind_batched(ctx, k, &p->line);
        if (!st && n == 4096) st = tc_plan_init(p);  // tensor-core tables (mfft_exec_c2c_tc)
    } else {
        st = fourstep_plan_init(p);
    }
    if (st) {
        mfft_plan_destroy(p);
        return st;
    }
    *out = p;
    return MFFT_SUCCESS;
}

extern "C" int mfft_plan_destroy(mfft_plan* plan) {
    if (!plan) return MFFT_SUCCESS;
    DeviceGuard g(plan->ctx->device);
    fourstep_plan_release(plan);
    tc_plan_release(plan);
    delete plan;
    return MFFT_SUCCESS;
}

extern "C" int64_t mfft_plan_size(const mfft_plan* plan) { return plan ? plan->n : 0; }

// ---------------------------------------------------------------------------
// execution
// ---------------------------------------------------------------------------

namespace mfft {

int launch_c2c_device(mfft_plan* plan, const float2* in, float2* out, int64_t batch, int direction,
                      cudaStream_t s, int adjoint) {
    cudaError_t e;
    // the adjoint of one direction runs the other direction's kernel
    const bool inv = (direction == MFFT_INVERSE) != (adjoint != 0);
    if (plan->n <= MFFT_MAX_SINGLE_N) {
        const BatchedKernel* k = plan->line.k;
        e = (inv ? k->inv : k->fwd)(in, out, batch, plan->line.tw, plan->ctx->dev_err, s, adjoint);
        if (e != cudaSuccess) return cuda_error(e, "batched FFT launch");
        return MFFT_SUCCESS;
    }
    return fourstep_exec(plan, in, out, batch, inv ? MFFT_INVERSE : MFFT_FORWARD, s, adjoint);
}

int check_exec_args(const void* in, void* out, int64_t batch, int direction, int flags) {
    if (batch < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, batch, -1, "batch must be >= 0, got %lld", (long long)batch);
    if (direction != MFFT_FORWARD && direction != MFFT_INVERSE)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "direction must be -1 or +1, got %d", direction);
    if (flags != MFFT_HOST_MEMORY && flags != MFFT_DEVICE_MEMORY)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown flags %d", flags);
    if (batch > 0 && (!in || !out)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL buffer");
    // the kernels move 16-byte chunks (bulk copies, cp.async, vector stores)
    if (flags == MFFT_DEVICE_MEMORY && (((uintptr_t)in | (uintptr_t)out) & 15))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "device buffers must be 16-byte aligned");
    return MFFT_SUCCESS;
}

// Reads and clears the context's device error word (set by a kernel whose
// bounded wait gave up).  Synchronous.
int check_device_error(mfft_ctx* ctx) {
    int code = 0;
    cudaError_t e = cudaMemcpy(&code, ctx->dev_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(e, "device error word");
    if (code) {
        cudaMemset(ctx->dev_err, 0, sizeof(int));
        return set_error(MFFT_ERR_TIMEOUT, -1, -1, -1,
                         "a device-side wait timed out (code %d); results of the call are invalid", code);
    }
    return MFFT_SUCCESS;
}

// Host-array call: stage through one device buffer on the context stream and
// wait, like MetalFFT's copy-in / commitAndWait / copy-out.
// the context's device pool: keeps what it has reserved between calls, so a
// repeated host-array call does not map and unmap its buffers every time
static int ctx_pool(mfft_ctx* ctx, cudaMemPool_t* out) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->pool) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx->device;
        cudaMemPool_t p = nullptr;
        cudaError_t e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess) return cuda_error(e, "device memory pool");
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        ctx->pool = p;
    }
    *out = ctx->pool;
    return MFFT_SUCCESS;
}

int run_host_staged(mfft_ctx* ctx, const void* in, void* out, size_t in_bytes, size_t out_bytes,
                    const std::function<int(void* d_in, void* d_out, cudaStream_t)>& body, bool in_place) {
    cudaStream_t s = ctx->stream;
    void* d_in = nullptr;
    void* d_out = nullptr;
    cudaMemPool_t pool = nullptr;
    int pst = ctx_pool(ctx, &pool);
    if (pst) return pst;
    cudaError_t e = cudaMallocFromPoolAsync(&d_in, in_bytes ? in_bytes : 16, pool, s);
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "Device buffer allocation failed: %s", cudaGetErrorString(e));
    const bool same = in_place && (in_bytes == out_bytes);
    if (same) {
        d_out = d_in;
    } else {
        e = cudaMallocFromPoolAsync(&d_out, out_bytes ? out_bytes : 16, pool, s);
        if (e != cudaSuccess) {
            cudaFreeAsync(d_in, s);
            cudaStreamSynchronize(s);
            return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "Device buffer allocation failed: %s", cudaGetErrorString(e));
        }
    }
    int st = MFFT_SUCCESS;
    if (in_bytes) e = cudaMemcpyAsync(d_in, in, in_bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) st = cuda_error(e, "host to device copy");
    if (!st) st = body(d_in, d_out, s);
    if (!st && out_bytes) {
        e = cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) st = cuda_error(e, "device to host copy");
    }
    cudaFreeAsync(d_in, s);
    if (!same) cudaFreeAsync(d_out, s);
    e = cudaStreamSynchronize(s);
    if (!st && e != cudaSuccess) st = cuda_error(e, "execution");
    if (!st) st = check_device_error(ctx);
    return st;
}

// Parallel memcpy on a fixed pool of host threads: copy() splits a copy into
// one part per worker (and one for the caller) and returns when all are done.
struct HostCopier {
    explicit HostCopier(int workers) {
        for (int i = 0; i < workers; ++i) th_.emplace_back([this, i] { run(i); });
    }
    ~HostCopier() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    void copy(void* dst, const void* src, size_t bytes) {
        const int parts = (int)th_.size() + 1;
        if (bytes < ((size_t)1 << 20) || parts == 1) {
            memcpy(dst, src, bytes);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            dst_ = (char*)dst;
            src_ = (const char*)src;
            bytes_ = bytes;
            parts_ = parts;
            pending_ = (int)th_.size();
            ++gen_;
        }
        cv_.notify_all();
        part(parts - 1);
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [this] { return pending_ == 0; });
    }

   private:
    void part(int i) {
        // 4 KiB-aligned split points
        const size_t step = ((bytes_ / parts_) + 4095) & ~(size_t)4095;
        const size_t a = step * (size_t)i, b = a + step < bytes_ ? a + step : bytes_;
        if (a < b) memcpy(dst_ + a, src_ + a, b - a);
    }
    void run(int i) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            part(i);
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    bool stop_ = false;
    uint64_t gen_ = 0;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t bytes_ = 0;
    int parts_ = 1, pending_ = 0;
};

void host_copier_free(HostCopier* c) { delete c; }

// host memory the driver cannot DMA from directly (not page-locked)
static bool pageable(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // (older drivers report unregistered memory as an error)
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

static int hstage_init(mfft_ctx* ctx) {
    if (ctx->hstage) return MFFT_SUCCESS;
    cudaError_t e = cudaHostAlloc(&ctx->hstage, STAGE_SLOT_BYTES * 2 * STAGE_SLOTS, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        ctx->hstage = nullptr;
        return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "pinned host staging: %s", cudaGetErrorString(e));
    }
    if (!ctx->copier) {
        const unsigned hw = std::thread::hardware_concurrency();
        ctx->copier = new HostCopier((int)(hw >= 16 ? 7 : hw >= 4 ? hw / 2 - 1 : 0));
    }
    return MFFT_SUCCESS;
}

static int stage_init(mfft_ctx* ctx) {
    if (ctx->h2d) return MFFT_SUCCESS;
    cudaError_t e = cudaMalloc(&ctx->stage, STAGE_SLOT_BYTES * 2 * STAGE_SLOTS);
    if (e != cudaSuccess) {
        ctx->stage = nullptr;
        return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "staging slots: %s", cudaGetErrorString(e));
    }
    cudaStream_t a = nullptr, b = nullptr;
    e = cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking);
    for (int i = 0; i < STAGE_SLOTS && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&ctx->ev_up[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_done[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_down[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        if (a) cudaStreamDestroy(a);
        if (b) cudaStreamDestroy(b);
        for (int i = 0; i < STAGE_SLOTS; ++i) {
            if (ctx->ev_up[i]) cudaEventDestroy(ctx->ev_up[i]);
            if (ctx->ev_done[i]) cudaEventDestroy(ctx->ev_done[i]);
            if (ctx->ev_down[i]) cudaEventDestroy(ctx->ev_down[i]);
            ctx->ev_up[i] = ctx->ev_done[i] = ctx->ev_down[i] = nullptr;
        }
        cudaFree(ctx->stage);
        ctx->stage = nullptr;
        return cuda_error(e, "staging streams");
    }
    ctx->h2d = a;
    ctx->d2h = b;
    return MFFT_SUCCESS;
}

int run_host_lines(mfft_ctx* ctx, const void* in, void* out, int64_t lines, size_t in_line, size_t out_line,
                   const std::function<int(const void* d_in, void* d_out, int64_t lines, cudaStream_t)>& body,
                   bool in_place, bool pair) {
    const size_t line_max = in_line > out_line ? in_line : out_line;
    int64_t per = line_max ? (int64_t)(STAGE_SLOT_BYTES / line_max) : lines;
    if (pair) per &= ~(int64_t)1;
    if (per < 1 || lines <= per)
        return run_host_staged(
            ctx, in, out, (size_t)lines * in_line, (size_t)lines * out_line,
            [&](void* di, void* dout, cudaStream_t s) { return body(di, dout, lines, s); }, in_place);
    std::lock_guard<std::mutex> lk(ctx->stage_mu);
    int st = stage_init(ctx);
    if (st) return st;
    // Pageable host arrays (what a Swift or numpy array is) go through pinned
    // host slots: the driver would otherwise stage each copy itself,
    // synchronously and on one thread, and the chunks would not overlap.
    const bool stage_host = pageable(in) || pageable(out);
    if (stage_host) {
        st = hstage_init(ctx);
        if (st) return st;
    }
    cudaStream_t sc = ctx->stream, sh = ctx->h2d, sd = ctx->d2h;
    char* slot = (char*)ctx->stage;
    char* hslot = (char*)ctx->hstage;
    cudaError_t e = cudaSuccess;
    // uploads start after the compute stream's earlier work (the slots may
    // still be read by the previous call's last transforms)
    e = cudaEventRecord(ctx->ev_done[0], sc);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sh, ctx->ev_done[0], 0);
    const int64_t nch = (lines + per - 1) / per;
    // pageable output: chunk c's result leaves its pinned slot for the
    // caller's array once its download is done
    auto drain = [&](int64_t c) {
        const int k = (int)(c % STAGE_SLOTS);
        const int64_t l0 = c * per, nl = lines - l0 < per ? lines - l0 : per;
        cudaError_t es = cudaEventSynchronize(ctx->ev_down[k]);
        if (es != cudaSuccess) return es;
        ctx->copier->copy((char*)out + (size_t)l0 * out_line, hslot + ((size_t)k * 2 + 1) * STAGE_SLOT_BYTES,
                          (size_t)nl * out_line);
        return cudaSuccess;
    };
    for (int64_t c = 0; c < nch && e == cudaSuccess && !st; ++c) {
        const int k = (int)(c % STAGE_SLOTS);
        const int64_t l0 = c * per, nl = lines - l0 < per ? lines - l0 : per;
        char* din = slot + (size_t)k * 2 * STAGE_SLOT_BYTES;
        char* dout = in_place ? din : din + STAGE_SLOT_BYTES;
        const char* src = (const char*)in + (size_t)l0 * in_line;
        if (stage_host) {
            // the pinned slots of chunk c - STAGE_SLOTS are free once its
            // download is done and its result copied out
            if (c >= STAGE_SLOTS) e = drain(c - STAGE_SLOTS);
            if (e != cudaSuccess) break;
            char* hin = hslot + (size_t)k * 2 * STAGE_SLOT_BYTES;
            ctx->copier->copy(hin, src, (size_t)nl * in_line);
            src = hin;
        }
        // slot k is free once the download of chunk c - STAGE_SLOTS is done
        if (c >= STAGE_SLOTS) e = cudaStreamWaitEvent(sh, ctx->ev_down[k], 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(din, src, (size_t)nl * in_line, cudaMemcpyHostToDevice, sh);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_up[k], sh);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sc, ctx->ev_up[k], 0);
        if (e != cudaSuccess) break;
        st = body(din, dout, nl, sc);
        if (st) break;
        e = cudaEventRecord(ctx->ev_done[k], sc);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sd, ctx->ev_done[k], 0);
        char* dst = stage_host ? hslot + ((size_t)k * 2 + 1) * STAGE_SLOT_BYTES : (char*)out + (size_t)l0 * out_line;
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, dout, (size_t)nl * out_line, cudaMemcpyDeviceToHost, sd);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_down[k], sd);
    }
    if (stage_host && !st && e == cudaSuccess)
        for (int64_t c = nch > STAGE_SLOTS ? nch - STAGE_SLOTS : 0; c < nch && e == cudaSuccess; ++c) e = drain(c);
    if (!st && e != cudaSuccess) st = cuda_error(e, "staged copies");
    cudaError_t e1 = cudaStreamSynchronize(sh), e2 = cudaStreamSynchronize(sc), e3 = cudaStreamSynchronize(sd);
    if (!st && e1 != cudaSuccess) st = cuda_error(e1, "execution");
    if (!st && e2 != cudaSuccess) st = cuda_error(e2, "execution");
    if (!st && e3 != cudaSuccess) st = cuda_error(e3, "execution");
    if (!st) st = check_device_error(ctx);
    return st;
}

}  // namespace mfft

extern "C" int mfft_exec_c2c(mfft_plan* plan, const void* in, void* out, int64_t batch, int direction,
                             int flags, void* stream) {
    if (!plan) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    int st = check_exec_args(in, out, batch, direction, flags);
    if (st) return st;
    if (batch == 0) return MFFT_SUCCESS;
    DeviceGuard g(plan->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY)
        return launch_c2c_device(plan, (const float2*)in, (float2*)out, batch, direction,
                                 (cudaStream_t)stream);
    const size_t line = (size_t)plan->n * sizeof(float2);
    return run_host_lines(
        plan->ctx, in, out, batch, line, line,
        [&](const void* di, void* dout, int64_t nl, cudaStream_t s) {
            return launch_c2c_device(plan, (const float2*)di, (float2*)dout, nl, direction, s);
        },
        true);
}

// Adjoint of mfft_exec_c2c (no reference counterpart): the same kernels with
// the direction swapped and the 1/n scale moved to the other side.
extern "C" int mfft_exec_c2c_backward(mfft_plan* plan, const void* grad_out, void* grad_in, int64_t batch,
                                      int direction, int flags, void* stream) {
    if (!plan) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    int st = check_exec_args(grad_out, grad_in, batch, direction, flags);
    if (st) return st;
    if (batch == 0) return MFFT_SUCCESS;
    DeviceGuard g(plan->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY)
        return launch_c2c_device(plan, (const float2*)grad_out, (float2*)grad_in, batch, direction,
                                 (cudaStream_t)stream, 1);
    const size_t line = (size_t)plan->n * sizeof(float2);
    return run_host_lines(
        plan->ctx, grad_out, grad_in, batch, line, line,
        [&](const void* di, void* dout, int64_t nl, cudaStream_t s) {
            return launch_c2c_device(plan, (const float2*)di, (float2*)dout, nl, direction, s, 1);
        },
        true);
}

// ---------------------------------------------------------------------------
// failure-path self-test
// ---------------------------------------------------------------------------

namespace {

// Waits, through the same bounded helper the pipelines use, on phase 0 of an
// mbarrier that expects one arrival nobody makes; gives up after limit_ns and
// records DEV_ERR_TMA_TIMEOUT in the context's error word.
__global__ void k_selftest_wait(int* dev_err, unsigned long long limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mfft::mbar_init(&bar, 1);
        mfft::fence_proxy_async_smem();
    }
    __syncthreads();
    if (!mfft::mbar_wait(&bar, 0, limit_ns) && threadIdx.x == 0)
        mfft::report_device_error(dev_err, mfft::DEV_ERR_TMA_TIMEOUT);
}

}  // namespace

extern "C" int mfft_selftest_bounded_wait(mfft_ctx* ctx, int64_t limit_ns) {
    if (!ctx) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "ctx is NULL");
    if (limit_ns < 1000 || limit_ns > 1000000000LL)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, limit_ns, -1, "limit_ns must be in [1e3, 1e9]");
    DeviceGuard g(ctx->device);
    k_selftest_wait<<<1, 32, 0, ctx->stream>>>(ctx->dev_err, (unsigned long long)limit_ns);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(e, "self-test launch");
    return check_device_error(ctx);
}
