// multi.cu -- FFTs of mixed sizes in ONE persistent launch of the queue
// kernel (fsqueue.h/.cu), driven by a device-side descriptor queue.
//
// No reference counterpart (MetalFFT.forward(batch:) takes one size; its
// four-step path even loops one command buffer per element,
// Sources/MetalFFT/FFT/MetalFFT.swift:198-202).  Here the host turns the size
// classes once into one array of 4096-point work items, in ticket order:
//   COLS  the column items of every four-step transform (n >= 8192),
//         transform by transform;
//   LINES the whole-line items (n <= 4096, 4096/n lines each);
//   ROWS  the row items of every four-step transform, in the same order.
// Each call zeroes the queue's counters and launches the kernel once: CTAs
// draw items by atomic ticket; a ROWS item starts when its transform's COLS
// items have been counted done (bounded wait), and the LINES items between
// the two phases keep the CTAs busy while the last columns finish.
// Four-step classes of 2^16 .. 2^20 points (up to FSQ_MAX_GROUPS of them) move
// their tiles by TMA inside the same launch: their transforms sit back to
// back, so one set of tensor maps per class covers them.
#include <algorithm>
#include <vector>

#include "capi_internal.h"
#include "fft_common.cuh"
#include "fsqueue.h"

using namespace mfft;

struct mfft_multi {
    mfft_ctx* ctx = nullptr;
    int64_t points = 0;
    FsqItem* d_items = nullptr;  // the queue, in ticket order
    FsqXform* d_xf = nullptr;
    int* d_counters = nullptr;   // ticket + one COLS count per four-step transform
    float2* scratch = nullptr;   // every four-step intermediate
    int nitems = 0, nxf = 0;
    FsqTables tabs{};
    std::vector<float2*> tables;  // owned four-step W_n tables
    struct Group {                // a four-step class whose tiles move by TMA
        int64_t offset, count;
        int logn, l1;
        long long scratch;
    };
    std::vector<Group> groups;
};

extern "C" int mfft_multi_destroy(mfft_multi* m) {
    if (!m) return MFFT_SUCCESS;
    DeviceGuard g(m->ctx->device);
    cudaFree(m->d_items);
    cudaFree(m->d_xf);
    cudaFree(m->d_counters);
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
                it.grp = -1;
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
        const int l1 = fourstep_split_for(ctx, logn);
        int grp = -1;
        if (fsq_tma_split(logn, l1) && (int)m->groups.size() < FSQ_MAX_GROUPS) {
            grp = (int)m->groups.size();
            m->groups.push_back(mfft_multi::Group{d.offset, d.count, logn, l1, scratch_pts});
        }
        const int nc = fsq_cols_items(logn), nr = fsq_rows_items(logn);
        for (int64_t j = 0; j < d.count; ++j) {
            const int id = (int)xfs.size();
            FsqXform x{};
            x.off = d.offset + j * d.n;
            x.scratch = scratch_pts;
            x.logn = logn;
            x.l1 = l1;
            scratch_pts += d.n;
            xfs.push_back(x);
            for (int c = 0; c < nc; ++c)
                cols.push_back(FsqItem{FSQ_COLS, logn, c, id, 0, 0, grp, x.off, x.scratch, l1, {0, 0, 0}});
            for (int r = 0; r < nr; ++r)
                rows.push_back(FsqItem{FSQ_ROWS, logn, r, id, 0, 0, grp, x.off, x.scratch, l1, {0, 0, 0}});
        }
    }
    if (st) {
        mfft_multi_destroy(m);
        return st;
    }
    std::vector<FsqItem> q = cols;
    q.insert(q.end(), lines.begin(), lines.end());
    q.insert(q.end(), rows.begin(), rows.end());
    if (q.size() > 0x3fffffff || xfs.size() > 0x3fffffff) {
        mfft_multi_destroy(m);
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "too many work items");
    }
    m->nitems = (int)q.size();
    m->nxf = (int)xfs.size();
    cudaError_t e = cudaSuccess;
    if (!q.empty()) e = cudaMalloc(&m->d_items, sizeof(FsqItem) * q.size());
    if (e == cudaSuccess && !xfs.empty()) e = cudaMalloc(&m->d_xf, sizeof(FsqXform) * xfs.size());
    if (e == cudaSuccess) e = cudaMalloc(&m->d_counters, sizeof(int) * (1 + xfs.size()));
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

// One memset of the queue counters and one launch.  The tensor maps of the
// TMA classes depend on the buffers, so they are encoded per call (host work,
// baked into a captured graph like any kernel argument).
static int multi_device(mfft_multi* m, const float2* in, float2* out, int direction, cudaStream_t s) {
    if (m->nitems == 0) return MFFT_SUCCESS;
    FsqQueueArgs q{};
    q.a.in = in;
    q.a.out = out;
    q.a.scratch = m->scratch;
    q.a.items = m->d_items;
    q.a.xf = m->d_xf;
    q.a.nitems = m->nitems;
    q.a.tabs = m->tabs;
    q.counters = m->d_counters;
    q.ngroups = (int)m->groups.size();
    for (int gi = 0; gi < q.ngroups; ++gi) {
        const auto& g = m->groups[gi];
        int n1, n2;
        fsq_split(g.logn, &n1, &n2, g.l1);
        const int C = FSQ_POINTS / n1, RW = FSQ_POINTS / n2;
        q.groups[gi] = FsqGroup{g.offset, g.scratch, g.logn, g.l1};
        FsqGroupMaps& mp = q.maps[gi];
        if (!encode_rows(&mp.ld, in + g.offset, (uint64_t)g.count * n1, n2, C) ||
            !encode_rows(&mp.stc, m->scratch + g.scratch, (uint64_t)g.count * n1, n2, C) ||
            !encode_rows(&mp.str, out + g.offset, (uint64_t)g.count * n2, n1, RW))
            return set_error(MFFT_ERR_LIBRARY_BUILD, -1, -1, -1, "mixed-size tensor maps could not be encoded");
    }
    cudaError_t e = cudaMemsetAsync(m->d_counters, 0, sizeof(int) * (1 + m->nxf), s);
    if (e == cudaSuccess) e = fsq_launch_queue(q, direction == MFFT_INVERSE, m->ctx->sms, m->ctx->dev_err, s);
    if (e != cudaSuccess) return cuda_error(e, "mixed-size launch");
    return MFFT_SUCCESS;
}

extern "C" int mfft_multi_exec(mfft_multi* m, const void* in, void* out, int direction, int flags, void* stream) {
    if (!m) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "multi is NULL");
    int st = check_exec_args(in, out, m->points, direction, flags);
    if (st) return st;
    // in == out is safe: a transform's ROWS items, which write its output,
    // start only after all of its COLS items have read its input; LINES items
    // read and write the same elements.
    DeviceGuard g(m->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY)
        return multi_device(m, (const float2*)in, (float2*)out, direction, (cudaStream_t)stream);
    const size_t bytes = (size_t)m->points * sizeof(float2);
    return run_host_staged(
        m->ctx, in, out, bytes, bytes,
        [&](void* di, void* dout, cudaStream_t s) { return multi_device(m, (const float2*)di, (float2*)dout, direction, s); },
        true);
}
