// multi.cu -- FFTs of mixed sizes in one persistent launch driven by a
// device-side work queue.
//
// No reference counterpart (MetalFFT.forward(batch:) takes one size; its
// four-step path even loops one command buffer per element,
// Sources/MetalFFT/FFT/MetalFFT.swift:198-202).  Here every work item is
// 16384 complex points, so one CTA shape (1024 threads, radix-16, one CTA per
// SM) serves every size:
//   kind LINES  16384/n whole lines of one size n <= 16384
//   kind COLS   one column tile (16384/n1 columns x n1 rows) of a four-step
//               transform n = n1*n2 > 16384: column FFTs + W_n twiddle -> scratch
//   kind ROWS   one row group (16384/n2 rows) of that transform: row FFTs,
//               transposed store to the output (needs all its COLS items done)
// CTAs take items in queue order with one atomicAdd.  A transform's ROWS
// items sit one transform behind its COLS items, so when a CTA reaches them
// the columns are normally finished and the 8 MiB intermediate is still in
// L2; a CTA that finds them unfinished waits on the transform's counter with a
// time limit (no item ever waits on a later item, so the wait ends), and on
// timeout records an error and skips the item.
#include <algorithm>
#include <vector>

#include "capi_internal.h"
#include "stockham.cuh"
#include "tma.cuh"

namespace mfft {

namespace {

constexpr int MQ_THREADS = 1024;
constexpr int MQ_POINTS = 16384;
constexpr int MQ_E = 16;
constexpr int MQ_SMEM = spad_size(MQ_POINTS) * 8;  // 139264 bytes, enough for every layout

enum : int { ITEM_LINES = 0, ITEM_COLS = 1, ITEM_ROWS = 2 };

struct Item {
    int kind;
    int logn;       // log2 of the line size (LINES) or of the transform size
    int index;      // COLS: tile, ROWS: row group
    int xform;      // four-step transform id (COLS / ROWS)
    long long off;  // LINES: element offset of the first line
    int lines;      // LINES: lines in this item
    int pad;
};

struct Xform {
    long long off;      // element offset of the transform in in/out
    long long scratch;  // element offset of its intermediate in scratch
    int logn, n1, n2;
    int ncols;          // number of COLS items
};

struct Tables {
    const float2* line_tw[9];  // n = 64 .. 16384 (E = 16 rows)
    const float2* fine[6];     // four-step n = 2^15 .. 2^20
    const float2* coarse[6];
};

template <int N, bool INV>
__device__ __forceinline__ void mq_lines(const float2* __restrict__ in, float2* __restrict__ out, long long off,
                                         int lines, const float2* __restrict__ tw, float2* smem) {
    constexpr int T = N / MQ_E;
    constexpr int FPB = MQ_POINTS / N;
    static_assert(T * FPB == MQ_THREADS, "one item fills the CTA");
    const int lf = threadIdx.x / T, t = threadIdx.x % T;
    const bool ok = lf < lines;
    float2 v[MQ_E];
    const float2* src = in + off + (long long)lf * N + t;
#pragma unroll
    for (int m = 0; m < MQ_E; ++m) {
        v[m] = ok ? __ldcs(src + m * T) : make_float2(0.f, 0.f);
        if constexpr (INV) v[m].y = -v[m].y;
    }
    fft_regs<N, MQ_E, (T <= 32)>(v, t, PadLine{smem + lf * spad_size(N)}, tw);
    if (ok) {
        float2* dst = out + off + (long long)lf * N + t;
        const float s = INV ? 1.0f / (float)N : 1.0f;
#pragma unroll
        for (int m = 0; m < MQ_E; ++m)
            __stcs(dst + m * T, INV ? make_float2(v[m].x * s, -v[m].y * s) : v[m]);
    }
}

template <int L, bool INV>
__device__ __forceinline__ void mq_cols(const float2* __restrict__ in, float2* __restrict__ mid, int n2, int tile,
                                        const float2* __restrict__ tw, const float2* __restrict__ fine,
                                        const float2* __restrict__ coarse, float2* smem) {
    constexpr int T = L / MQ_E;
    constexpr int C = MQ_POINTS / L;  // columns per item
    const int c = threadIdx.x % C, t = threadIdx.x / C;
    const int col = tile * C + c;
    float2 v[MQ_E];
#pragma unroll
    for (int m = 0; m < MQ_E; ++m) {
        v[m] = __ldcs(in + (size_t)(t + m * T) * n2 + col);
        if constexpr (INV) v[m].y = -v[m].y;
    }
    fft_regs<L, MQ_E, false>(v, t, SwzLine<C>{smem, c}, tw);
#pragma unroll
    for (int m = 0; m < MQ_E; ++m) {
        const unsigned k1 = (unsigned)(t + m * T);
        const unsigned e = (unsigned)col * k1;
        const float2 w = cmul(__ldg(fine + (e & 1023u)), __ldg(coarse + (e >> 10)));
        mid[(size_t)k1 * n2 + col] = cmul(v[m], w);
    }
}

template <int L, bool INV>
__device__ __forceinline__ void mq_rows(const float2* __restrict__ mid, float2* __restrict__ out, int n1, int group,
                                        const float2* __restrict__ tw, float2* smem) {
    constexpr int T = L / MQ_E;
    constexpr int RW = MQ_POINTS / L;  // rows per item
    const int row0 = group * RW;
    const float4* src = reinterpret_cast<const float4*>(mid + (size_t)row0 * L);
    for (int q = threadIdx.x; q < RW * L / 2; q += MQ_THREADS) {
        const float4 x = __ldcg(src + q);
        const int e = 2 * q, r = e / L, i = e % L;
        SwzLine<RW> line{smem, r};
        line[i] = make_float2(x.x, x.y);
        line[i + 1] = make_float2(x.z, x.w);
    }
    __syncthreads();
    const int r = threadIdx.x % RW, t = threadIdx.x / RW;
    const SwzLine<RW> line{smem, r};
    float2 v[MQ_E];
#pragma unroll
    for (int m = 0; m < MQ_E; ++m) v[m] = line[t + m * T];
    __syncthreads();
    fft_regs<L, MQ_E, false>(v, t, line, tw);
    const float s = INV ? 1.0f / (float)((size_t)n1 * L) : 1.0f;
#pragma unroll
    for (int m = 0; m < MQ_E; ++m) {
        float2 y = v[m];
        if constexpr (INV) y = make_float2(y.x * s, -y.y * s);
        __stcs(out + (size_t)(t + m * T) * n1 + row0 + r, y);
    }
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <bool INV>
__global__ void __launch_bounds__(MQ_THREADS, 1)
    k_multi(const float2* __restrict__ in, float2* __restrict__ out, float2* __restrict__ scratch,
            const Item* __restrict__ items, int nitems, const Xform* __restrict__ xf, int* counters, Tables tabs,
            int* dev_err) {
    extern __shared__ __align__(16) float2 smem[];
    __shared__ int item_sh;
    int* head = counters;         // counters[0]: next item
    int* cols_done = counters + 1;  // counters[1 + j]: finished COLS items of transform j
    for (;;) {
        if (threadIdx.x == 0) item_sh = atomicAdd(head, 1);
        __syncthreads();
        const int id = item_sh;
        __syncthreads();  // item_sh read by all; smem free from the previous item
        if (id >= nitems) break;
        const Item it = items[id];
        if (it.kind == ITEM_LINES) {
            const float2* tw = tabs.line_tw[it.logn - 6];
            switch (it.logn) {
                case 6: mq_lines<64, INV>(in, out, it.off, it.lines, tw, smem); break;
                case 7: mq_lines<128, INV>(in, out, it.off, it.lines, tw, smem); break;
                case 8: mq_lines<256, INV>(in, out, it.off, it.lines, tw, smem); break;
                case 9: mq_lines<512, INV>(in, out, it.off, it.lines, tw, smem); break;
                case 10: mq_lines<1024, INV>(in, out, it.off, it.lines, tw, smem); break;
                case 11: mq_lines<2048, INV>(in, out, it.off, it.lines, tw, smem); break;
                case 12: mq_lines<4096, INV>(in, out, it.off, it.lines, tw, smem); break;
                case 13: mq_lines<8192, INV>(in, out, it.off, it.lines, tw, smem); break;
                default: mq_lines<16384, INV>(in, out, it.off, it.lines, tw, smem); break;
            }
        } else {
            const Xform x = xf[it.xform];
            const int lc = ilog2c(x.n1) - 6, lr = ilog2c(x.n2) - 6;
            if (it.kind == ITEM_COLS) {
                const float2* fine = tabs.fine[x.logn - 15];
                const float2* coarse = tabs.coarse[x.logn - 15];
                const float2* src = in + x.off;
                float2* mid = scratch + x.scratch;
                const float2* tw = tabs.line_tw[lc];
                switch (x.n1) {
                    case 128: mq_cols<128, INV>(src, mid, x.n2, it.index, tw, fine, coarse, smem); break;
                    case 256: mq_cols<256, INV>(src, mid, x.n2, it.index, tw, fine, coarse, smem); break;
                    case 512: mq_cols<512, INV>(src, mid, x.n2, it.index, tw, fine, coarse, smem); break;
                    default: mq_cols<1024, INV>(src, mid, x.n2, it.index, tw, fine, coarse, smem); break;
                }
                __threadfence();
                __syncthreads();
                if (threadIdx.x == 0) atomicAdd(cols_done + it.xform, 1);
            } else {
                if (threadIdx.x == 0) {
                    int ok = 1;
                    if (ld_acquire(cols_done + it.xform) < x.ncols) {
                        const uint64_t t0 = globaltimer_ns();
                        while (ld_acquire(cols_done + it.xform) < x.ncols) {
                            if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
                                ok = 0;
                                break;
                            }
                            __nanosleep(256);
                        }
                    }
                    if (!ok) report_device_error(dev_err, DEV_ERR_QUEUE_TIMEOUT);
                    item_sh = ok;
                }
                __syncthreads();
                const bool ready = item_sh != 0;
                __syncthreads();
                if (ready) {
                    const float2* mid = scratch + x.scratch;
                    float2* dst = out + x.off;
                    const float2* tw = tabs.line_tw[lr];
                    switch (x.n2) {
                        case 256: mq_rows<256, INV>(mid, dst, x.n1, it.index, tw, smem); break;
                        case 512: mq_rows<512, INV>(mid, dst, x.n1, it.index, tw, smem); break;
                        default: mq_rows<1024, INV>(mid, dst, x.n1, it.index, tw, smem); break;
                    }
                }
            }
        }
    }
}

}  // namespace

}  // namespace mfft

using namespace mfft;

struct mfft_multi {
    mfft_ctx* ctx = nullptr;
    std::vector<mfft_multi_desc> descs;
    int64_t points = 0;
    Item* d_items = nullptr;
    Xform* d_xf = nullptr;
    int* d_counters = nullptr;
    float2* scratch = nullptr;
    int nitems = 0, nxf = 0;
    Tables tabs{};
    std::vector<mfft_plan*> fs_plans;  // own the four-step tables
};

extern "C" int mfft_multi_destroy(mfft_multi* m) {
    if (!m) return MFFT_SUCCESS;
    DeviceGuard g(m->ctx->device);
    cudaFree(m->d_items);
    cudaFree(m->d_xf);
    cudaFree(m->d_counters);
    cudaFree(m->scratch);
    for (auto* p : m->fs_plans) mfft_plan_destroy(p);
    delete m;
    return MFFT_SUCCESS;
}

extern "C" int64_t mfft_multi_points(const mfft_multi* m) { return m ? m->points : 0; }

extern "C" int mfft_multi_create(mfft_ctx* ctx, const mfft_multi_desc* descs, int ndesc, mfft_multi** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    *out = nullptr;
    if (ndesc < 0 || (ndesc > 0 && !descs)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "bad descriptors");
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    int64_t points = 0;
    for (int i = 0; i < ndesc; ++i) {
        const mfft_multi_desc& d = descs[i];
        if (!is_pow2_in(d.n, 64, MFFT_MAX_N))
            return set_error(MFFT_ERR_UNSUPPORTED_SIZE, d.n, -1, i, "Unsupported FFT size: %lld (descriptor %d)",
                             (long long)d.n, i);
        if (d.count < 0 || d.offset < 0)
            return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, i, "descriptor %d: negative count or offset", i);
        points = std::max<int64_t>(points, d.offset + d.n * d.count);
    }
    DeviceGuard g(ctx->device);
    mfft_multi* m = new mfft_multi();
    m->ctx = ctx;
    m->descs.assign(descs, descs + ndesc);
    m->points = points;
    int st = MFFT_SUCCESS;

    // line twiddles for every size (E = 16 rows), four-step tables per size
    for (int l = 6; l <= 14 && !st; ++l) {
        const BatchedKernel* bk = nullptr;
        int cnt = 0;
        const BatchedKernel* ks = batched_kernels(&cnt);
        for (int i = 0; i < cnt && !bk; ++i)
            if (ks[i].n == (1 << l) && ks[i].e == 16) bk = &ks[i];
        float2* tw = nullptr;
        st = ctx_twiddles(ctx, bk, &tw);
        m->tabs.line_tw[l - 6] = tw;
    }
    std::vector<Item> cols_items, rows_items, line_items;
    std::vector<Xform> xfs;
    long long scratch_pts = 0;
    for (int i = 0; i < ndesc && !st; ++i) {
        const mfft_multi_desc& d = descs[i];
        const int logn = ilog2c(d.n);
        if (d.n <= MFFT_MAX_SINGLE_N) {
            const int per = (int)(MQ_POINTS / d.n);
            for (int64_t l = 0; l < d.count; l += per) {
                Item it{};
                it.kind = ITEM_LINES;
                it.logn = logn;
                it.off = d.offset + l * d.n;
                it.lines = (int)std::min<int64_t>(per, d.count - l);
                line_items.push_back(it);
            }
        } else {
            if (d.count > 0 && !m->tabs.fine[logn - 15]) {
                mfft_plan* p = nullptr;
                st = mfft_plan_create(ctx, d.n, &p);
                if (st) break;
                m->fs_plans.push_back(p);
                m->tabs.fine[logn - 15] = p->fs.tables;
                m->tabs.coarse[logn - 15] = p->fs.tables + 1024;
            }
            const int n1 = 1 << (logn / 2), n2 = (int)(d.n / n1);
            for (int64_t j = 0; j < d.count; ++j) {
                Xform x{};
                x.off = d.offset + j * d.n;
                x.scratch = scratch_pts;
                x.logn = logn;
                x.n1 = n1;
                x.n2 = n2;
                x.ncols = n2 / (MQ_POINTS / n1);
                scratch_pts += d.n;
                const int id = (int)xfs.size();
                xfs.push_back(x);
                for (int c = 0; c < x.ncols; ++c) cols_items.push_back(Item{ITEM_COLS, logn, c, id, 0, 0, 0});
                for (int r = 0; r < n1 / (MQ_POINTS / n2); ++r) rows_items.push_back(Item{ITEM_ROWS, logn, r, id, 0, 0, 0});
            }
        }
    }
    if (st) {
        mfft_multi_destroy(m);
        return st;
    }
    // queue: COLS of transform j, then ROWS of transform j-1 (one behind), small
    // sizes after the four-step work (they fill the tail of the launch)
    std::vector<Item> q;
    size_t ci = 0, ri = 0;
    for (size_t j = 0; j < xfs.size(); ++j) {
        while (ci < cols_items.size() && cols_items[ci].xform == (int)j) q.push_back(cols_items[ci++]);
        if (j > 0)
            while (ri < rows_items.size() && rows_items[ri].xform == (int)j - 1) q.push_back(rows_items[ri++]);
    }
    while (ri < rows_items.size()) q.push_back(rows_items[ri++]);
    q.insert(q.end(), line_items.begin(), line_items.end());
    m->nitems = (int)q.size();
    m->nxf = (int)xfs.size();
    cudaError_t e = cudaSuccess;
    if (!q.empty()) e = cudaMalloc(&m->d_items, sizeof(Item) * q.size());
    if (e == cudaSuccess && !xfs.empty()) e = cudaMalloc(&m->d_xf, sizeof(Xform) * xfs.size());
    if (e == cudaSuccess) e = cudaMalloc(&m->d_counters, sizeof(int) * (1 + xfs.size()));
    if (e == cudaSuccess && scratch_pts) e = cudaMalloc(&m->scratch, sizeof(float2) * scratch_pts);
    if (e == cudaSuccess && !q.empty())
        e = cudaMemcpy(m->d_items, q.data(), sizeof(Item) * q.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !xfs.empty())
        e = cudaMemcpy(m->d_xf, xfs.data(), sizeof(Xform) * xfs.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(k_multi<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, MQ_SMEM);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_multi<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, MQ_SMEM);
    }
    if (e != cudaSuccess) {
        mfft_multi_destroy(m);
        return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "mixed-size queue: %s", cudaGetErrorString(e));
    }
    *out = m;
    return MFFT_SUCCESS;
}

static int multi_device(mfft_multi* m, const float2* in, float2* out, int direction, cudaStream_t s) {
    if (m->nitems == 0) return MFFT_SUCCESS;
    cudaError_t e = cudaMemsetAsync(m->d_counters, 0, sizeof(int) * (1 + m->nxf), s);
    if (e != cudaSuccess) return cuda_error(e, "queue reset");
    const int grid = std::min(m->ctx->sms, m->nitems);
    if (direction == MFFT_INVERSE)
        k_multi<true><<<grid, MQ_THREADS, MQ_SMEM, s>>>(in, out, m->scratch, m->d_items, m->nitems, m->d_xf,
                                                        m->d_counters, m->tabs, m->ctx->dev_err);
    else
        k_multi<false><<<grid, MQ_THREADS, MQ_SMEM, s>>>(in, out, m->scratch, m->d_items, m->nitems, m->d_xf,
                                                         m->d_counters, m->tabs, m->ctx->dev_err);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "mixed-size launch");
    return MFFT_SUCCESS;
}

extern "C" int mfft_multi_exec(mfft_multi* m, const void* in, void* out, int direction, int flags, void* stream) {
    if (!m) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "multi is NULL");
    int st = check_exec_args(in, out, m->points, direction, flags);
    if (st) return st;
    // in == out is safe: a ROWS item writes only its own transform, whose
    // input its COLS items consumed before it starts; LINES items read and
    // write the same elements.
    DeviceGuard g(m->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY)
        return multi_device(m, (const float2*)in, (float2*)out, direction, (cudaStream_t)stream);
    const size_t bytes = (size_t)m->points * sizeof(float2);
    return run_host_staged(
        m->ctx, in, out, bytes, bytes,
        [&](void* di, void* dout, cudaStream_t s) { return multi_device(m, (const float2*)di, (float2*)dout, direction, s); },
        true);
}
