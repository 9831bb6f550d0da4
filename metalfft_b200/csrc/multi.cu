// multi.cu -- FFTs of mixed sizes in one CUDA graph of at most two launches
// of the item kernel (fsqueue.h/.cu).
//
// No reference counterpart (MetalFFT.forward(batch:) takes one size; its
// four-step path even loops one command buffer per element,
// Sources/MetalFFT/FFT/MetalFFT.swift:198-202).  Here the host turns the size
// classes into two item lists of 4096 points per item:
//   pass 0   the COLS items of every four-step transform (n >= 8192), then
//            the whole-line items (n <= 4096, 4096/n lines each), which fill
//            the tail of the launch;
//   pass 1   the ROWS items of every four-step transform (absent when there
//            is none).
// Four-step classes of 2^16 .. 2^20 points skip the lists: their transforms
// are contiguous, so each class runs the uniform passes whose tiles move by
// TMA (fourstep.cu), its column pass after list pass 0 and its row pass after
// list pass 1.
#include <algorithm>
#include <vector>

#include "capi_internal.h"
#include "fft_common.cuh"
#include "fsqueue.h"

using namespace mfft;

struct mfft_multi {
    mfft_ctx* ctx = nullptr;
    int64_t points = 0;
    FsqItem* d_items = nullptr;  // pass 0 items, then pass 1 items
    FsqXform* d_xf = nullptr;
    float2* scratch = nullptr;   // every four-step intermediate
    int nitems0 = 0, nitems1 = 0;
    FsqTables tabs{};
    std::vector<float2*> tables;  // owned four-step W_n tables
    struct Group {                // a four-step class run by the TMA passes
        int64_t offset, count;
        int logn;
        long long scratch;
    };
    std::vector<Group> groups;
};

extern "C" int mfft_multi_destroy(mfft_multi* m) {
    if (!m) return MFFT_SUCCESS;
    DeviceGuard g(m->ctx->device);
    cudaFree(m->d_items);
    cudaFree(m->d_xf);
    cudaFree(m->scratch);
    for (float2* t : m->tables) cudaFree(t);
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
        if (d.offset & 1)
            return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, d.offset, i, "descriptor %d: offset must be even", i);
        points = std::max<int64_t>(points, d.offset + d.n * d.count);
    }
    DeviceGuard g(ctx->device);
    mfft_multi* m = new mfft_multi();
    m->ctx = ctx;
    m->points = points;
    int st = MFFT_SUCCESS;
    for (int l = 6; l <= 12 && !st; ++l) {
        float2* tw = nullptr;
        st = line_twiddles(ctx, 1 << l, &tw);
        m->tabs.line_tw[l - 6] = tw;
    }

    std::vector<FsqItem> lines, cols, rows;
    std::vector<FsqXform> xfs;
    long long scratch_pts = 0;
    for (int i = 0; i < ndesc && !st; ++i) {
        const mfft_multi_desc& d = descs[i];
        if (d.count == 0) continue;
        const int logn = ilog2c(d.n);
        if (d.n <= FSQ_POINTS) {
            const int per = (int)(FSQ_POINTS / d.n);
            for (int64_t l = 0; l < d.count; l += per) {
                FsqItem it{};
                it.kind = FSQ_LINES;
                it.logn = logn;
                it.off = d.offset + l * d.n;
                it.lines = (int)std::min<int64_t>(per, d.count - l);
                lines.push_back(it);
            }
            continue;
        }
        if (!m->tabs.fine[logn - 13]) {
            float2* t = nullptr;
            st = fourstep_tables(ctx, d.n, &t);
            if (st) break;
            m->tables.push_back(t);
            m->tabs.fine[logn - 13] = t;
            m->tabs.coarse[logn - 13] = t + 1024;
        }
        if (fsq_tma_size(logn)) {
            m->groups.push_back(mfft_multi::Group{d.offset, d.count, logn, scratch_pts});
            scratch_pts += d.n * d.count;
            continue;
        }
        const int nc = fsq_cols_items(logn), nr = fsq_rows_items(logn);
        for (int64_t j = 0; j < d.count; ++j) {
            const int id = (int)xfs.size();
            FsqXform x{};
            x.off = d.offset + j * d.n;
            x.scratch = scratch_pts;
            x.logn = logn;
            scratch_pts += d.n;
            xfs.push_back(x);
            for (int c = 0; c < nc; ++c) cols.push_back(FsqItem{FSQ_COLS, logn, c, id, 0, 0, 0});
            for (int r = 0; r < nr; ++r) rows.push_back(FsqItem{FSQ_ROWS, logn, r, id, 0, 0, 0});
        }
    }
    if (st) {
        mfft_multi_destroy(m);
        return st;
    }
    std::vector<FsqItem> q = cols;
    q.insert(q.end(), lines.begin(), lines.end());
    const size_t n0 = q.size();
    q.insert(q.end(), rows.begin(), rows.end());
    if (n0 > 0x7fffffff || rows.size() > 0x7fffffff) {
        mfft_multi_destroy(m);
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "too many work items");
    }
    m->nitems0 = (int)n0;
    m->nitems1 = (int)rows.size();
    cudaError_t e = cudaSuccess;
    if (!q.empty()) e = cudaMalloc(&m->d_items, sizeof(FsqItem) * q.size());
    if (e == cudaSuccess && !xfs.empty()) e = cudaMalloc(&m->d_xf, sizeof(FsqXform) * xfs.size());
    if (e == cudaSuccess && scratch_pts) e = cudaMalloc(&m->scratch, sizeof(float2) * scratch_pts);
    if (e == cudaSuccess && !q.empty())
        e = cudaMemcpy(m->d_items, q.data(), sizeof(FsqItem) * q.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !xfs.empty())
        e = cudaMemcpy(m->d_xf, xfs.data(), sizeof(FsqXform) * xfs.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = fsq_prepare();
    if (e != cudaSuccess) {
        mfft_multi_destroy(m);
        return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "mixed-size queue: %s", cudaGetErrorString(e));
    }
    *out = m;
    return MFFT_SUCCESS;
}

static int multi_device(mfft_multi* m, const float2* in, float2* out, int direction, cudaStream_t s) {
    FsqArgs a{};
    a.in = in;
    a.out = out;
    a.scratch = m->scratch;
    a.items = m->d_items;
    a.xf = m->d_xf;
    a.nitems = m->nitems0;
    a.tabs = m->tabs;
    const bool inv = direction == MFFT_INVERSE;
    cudaError_t e = fsq_launch(a, inv, m->ctx->sms, s);
    if (e != cudaSuccess) return cuda_error(e, "mixed-size launch");
    for (const auto& g : m->groups) {
        int st = fourstep_tma_pass(FSQ_COLS, m->tabs, in + g.offset, out + g.offset, m->scratch + g.scratch, g.count,
                                   g.logn, inv, m->ctx, s);
        if (st) return st;
    }
    if (m->nitems1) {
        a.items = m->d_items + m->nitems0;
        a.nitems = m->nitems1;
        e = fsq_launch(a, inv, m->ctx->sms, s);
        if (e != cudaSuccess) return cuda_error(e, "mixed-size launch");
    }
    for (const auto& g : m->groups) {
        int st = fourstep_tma_pass(FSQ_ROWS, m->tabs, in + g.offset, out + g.offset, m->scratch + g.scratch, g.count,
                                   g.logn, inv, m->ctx, s);
        if (st) return st;
    }
    return MFFT_SUCCESS;
}

extern "C" int mfft_multi_exec(mfft_multi* m, const void* in, void* out, int direction, int flags, void* stream) {
    if (!m) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "multi is NULL");
    int st = check_exec_args(in, out, m->points, direction, flags);
    if (st) return st;
    // in == out is safe: the row pass, which writes the four-step outputs,
    // starts after the column pass has read every input; LINES items read
    // and write the same elements.
    DeviceGuard g(m->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY)
        return multi_device(m, (const float2*)in, (float2*)out, direction, (cudaStream_t)stream);
    const size_t bytes = (size_t)m->points * sizeof(float2);
    return run_host_staged(
        m->ctx, in, out, bytes, bytes,
        [&](void* di, void* dout, cudaStream_t s) { return multi_device(m, (const float2*)di, (float2*)dout, direction, s); },
        true);
}
