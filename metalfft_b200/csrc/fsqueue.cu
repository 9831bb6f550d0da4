// fsqueue.cu -- the persistent item kernel (item kinds and passes in
// fsqueue.h).
//
// B200 form of the reference's batched and four-step dispatches
// (Sources/MetalFFT/FFT/MetalFFT.swift:159-277: one threadgroup per line, or
// five encoders and three scalar transposes per four-step transform, one
// command buffer per batch element).  Here one launch runs a whole pass:
//  * every item moves with 16-byte cp.async copies into the stage buffer the
//    CTA is not computing on, so DRAM traffic overlaps the FFT arithmetic;
//    the schedule is static, so the next item is always known and no CTA
//    ever waits for another;
//  * the row pass reads each intermediate once and then discards its lines
//    from L2 (discard.global.L2), so a dead intermediate still in L2 is never
//    written back to DRAM;
//  * the column tiles and the transposed row-pass output go through shared
//    memory in 16-byte chunks with an XOR swizzle on chunk pairs, so global
//    accesses are whole 32-byte sectors and shared-memory reads stay within
//    two wavefronts of the minimum.
// Each line transform is the in-register radix-16 Stockham FFT of
// stockham.cuh (padded exchange, one line, column or row per T = n/16
// threads, t fastest).
#include "fsqueue.h"
#include "stockham.cuh"
#include "tma.cuh"

namespace mfft {

namespace {

constexpr int QSTAGE = spad_size(FSQ_POINTS);  // float2 per stage buffer (4352)
constexpr int QSMEM = 2 * QSTAGE * (int)sizeof(float2);

__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// 16-byte global -> shared copy that bypasses L1 (streamed data is read once).
__device__ __forceinline__ void cp_async16(float2* sdst, const float2* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async16_hint(float2* sdst, const float2* gsrc, uint64_t pol) {
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(smem_u32(sdst)), "l"(gsrc),
                 "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void discard_l2_line(const void* p) {
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

// Element (row i, column c) of a tile 2^lw columns wide: rows are 2^lw
// consecutive slots, and the 16-byte column pairs of row i are permuted by
// XOR with the index of the 128-byte window row i starts in, so rows that
// would share banks when a warp walks down a column sit on different pairs.
__device__ __forceinline__ int pair_swz(int i, int lw) {
    const int sh = lw < 4 ? 4 - lw : 0;  // rows per 128 bytes = 2^sh
    return (i >> sh) & ((1 << (lw - 1)) - 1);
}
__device__ __forceinline__ int tidx(int i, int c, int lw) {
    return (i << lw) + ((((c >> 1) ^ pair_swz(i, lw)) << 1) | (c & 1));
}

// 2^lr rows x 2^lw columns of a row-major array (row stride `stride`) ->
// stage, in the tidx layout.
__device__ __forceinline__ void load_tile(float2* st, const float2* g, int lr, int lw, long long stride,
                                          uint64_t pol) {
    const int lp = lw - 1, pm = (1 << lp) - 1;
    const int chunks = 1 << (lr + lp);
    for (int q = threadIdx.x; q < chunks; q += FSQ_THREADS) {
        const int i = q >> lp, p = q & pm;
        cp_async16_hint(st + (i << lw) + ((p ^ pair_swz(i, lw)) << 1), g + i * stride + 2 * p, pol);
    }
}

template <bool STREAM>
__device__ __forceinline__ void store_tile(const float2* st, float2* g, int lr, int lw, long long stride) {
    const int lp = lw - 1, pm = (1 << lp) - 1;
    const int chunks = 1 << (lr + lp);
    for (int q = threadIdx.x; q < chunks; q += FSQ_THREADS) {
        const int i = q >> lp, p = q & pm;
        const float4 v = *reinterpret_cast<const float4*>(st + (i << lw) + ((p ^ pair_swz(i, lw)) << 1));
        float4* dst = reinterpret_cast<float4*>(g + i * stride + 2 * p);
        if constexpr (STREAM) __stcs(dst, v);
        else *dst = v;
    }
}

// `count` (even) contiguous points -> stage
__device__ __forceinline__ void load_linear(float2* st, const float2* g, int count, bool hint, uint64_t pol) {
    for (int q = threadIdx.x; q < count / 2; q += FSQ_THREADS) {
        if (hint) cp_async16_hint(st + 2 * q, g + 2 * q, pol);
        else cp_async16(st + 2 * q, g + 2 * q);
    }
}

// ---- the three item kinds ---------------------------------------------------

// Output scale of a transform of n points: the inverse is scaled by 1/n, the
// forward is not; the adjoint swaps the two (both scalings are exact).
template <bool INV>
__device__ __forceinline__ float out_scale(long long n, int adj) {
    return (INV != (adj != 0)) ? 1.0f / (float)n : 1.0f;
}

template <int L, bool INV>
__device__ __forceinline__ void do_lines(float2* st, float2* __restrict__ out, long long off, int lines,
                                         const float2* __restrict__ tw, float s) {
    constexpr int T = L / 16;
    const int u = threadIdx.x / T, t = threadIdx.x % T;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        v[m] = st[u * L + t + m * T];
        if constexpr (INV) v[m].y = -v[m].y;
    }
    __syncthreads();  // the raw item is in registers; the stage becomes the exchange area
    fft_regs<L, 16, (T <= 32)>(v, t, PadLineS{st + u * spad_size(L)}, tw);
    if (u < lines) {
        float2* dst = out + off + (long long)u * L + t;
#pragma unroll
        for (int m = 0; m < 16; ++m) __stcs(dst + m * T, make_float2(v[m].x * s, INV ? -v[m].y * s : v[m].y * s));
    }
}

__device__ __forceinline__ float2 tw_n(const float2* __restrict__ fine, const float2* __restrict__ coarse,
                                       unsigned e) {
    return cmul(__ldg(fine + (e & 1023u)), __ldg(coarse + (e >> 10)));
}

template <int L, bool INV, bool TILE_OUT = false>
__device__ __forceinline__ void do_cols(float2* st, float2* __restrict__ mid, int ln2, int col0,
                                        const float2* __restrict__ tw, const float2* __restrict__ fine,
                                        const float2* __restrict__ coarse) {
    constexpr int T = L / 16, C = FSQ_POINTS / L, LC = ilog2c(C), LL = ilog2c(L);
    const int c = threadIdx.x / T, t = threadIdx.x % T;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        v[m] = st[tidx(t + m * T, c, LC)];
        if constexpr (INV) v[m].y = -v[m].y;
    }
    __syncthreads();
    fft_regs<L, 16, (T <= 32)>(v, t, PadLineS{st + c * spad_size(L)}, tw);
    // W_n^{col*k1}, k1 = t + m*T: base W^{col*t} times W^{col*T*m}, the latter
    // a product of at most four of W^{col*T*{1,2,4,8}} (warp-uniform loads);
    // every exponent stays below n
    {
        const unsigned col = (unsigned)(col0 + c), step = col * (unsigned)T;
        const float2 base = tw_n(fine, coarse, col * (unsigned)t);
        const float2 s1 = tw_n(fine, coarse, step), s2 = tw_n(fine, coarse, 2 * step);
        const float2 s4 = tw_n(fine, coarse, 4 * step), s8 = tw_n(fine, coarse, 8 * step);
        float2 u[4];
        u[0] = base;
        u[1] = cmul(base, s1);
        u[2] = cmul(base, s2);
        u[3] = cmul(u[1], s2);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float2 w4 = cmul(u[q], s4);
            v[q] = cmul(v[q], u[q]);
            v[q + 8] = cmul(v[q + 8], cmul(u[q], s8));
            v[q + 4] = cmul(v[q + 4], w4);
            v[q + 12] = cmul(v[q + 12], cmul(w4, s8));
        }
    }
    __syncthreads();  // every exchange read is done before the output tile overwrites the stage
#pragma unroll
    for (int m = 0; m < 16; ++m) st[tidx(t + m * T, c, LC)] = v[m];
    if constexpr (!TILE_OUT) {  // (the TMA caller fences and synchronises before its bulk store)
        __syncthreads();
        store_tile<false>(st, mid + col0, LL, LC, 1LL << ln2);
    }
}

template <int L, bool INV, bool TILE_OUT = false>
__device__ __forceinline__ void do_rows(float2* st, const float2* mid_rows, float2* __restrict__ out, int ln1,
                                        int row0, const float2* __restrict__ tw, float scale) {
    constexpr int T = L / 16, RW = FSQ_POINTS / L, LR = ilog2c(RW), LL = ilog2c(L);
    const int r = threadIdx.x / T, t = threadIdx.x % T;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = st[r * L + t + m * T];
    // the intermediate rows now live on chip: drop them from L2 without a
    // write-back (32 KiB = 256 lines of 128 bytes, one per thread)
    discard_l2_line(reinterpret_cast<const char*>(mid_rows) + 128 * threadIdx.x);
    __syncthreads();
    fft_regs<L, 16, (T <= 32)>(v, t, PadLineS{st + r * spad_size(L)}, tw);
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 16; ++m)
        st[tidx(t + m * T, r, LR)] = make_float2(v[m].x * scale, INV ? -v[m].y * scale : v[m].y * scale);
    if constexpr (!TILE_OUT) {
        __syncthreads();
        store_tile<true>(st, out + row0, LL, LR, 1LL << ln1);
    }
}

// ---- items ----------------------------------------------------------------------

struct Work {
    int kind, logn, index, lines, l1;
    long long off;      // LINES: first line; COLS / ROWS: the transform in in / out
    long long scratch;  // COLS / ROWS: the transform's intermediate
};

__device__ __forceinline__ Work get_work(const FsqArgs& a, int p) {
    Work w;
    if (a.items) {
        const FsqItem it = a.items[p];
        w.kind = it.kind;
        w.logn = it.logn;
        w.index = it.index;
        w.lines = it.lines;
        w.off = it.off;
        w.scratch = 0;
        w.l1 = it.l1;
        if (it.kind != FSQ_LINES) {
            const FsqXform x = a.xf[it.xform];
            w.off = x.off;
            w.scratch = x.scratch;
        }
        return w;
    }
    const unsigned j = (unsigned)p / (unsigned)a.u_per;
    w.kind = a.u_kind;
    w.logn = a.u_logn;
    w.index = p - (int)(j * (unsigned)a.u_per);
    w.lines = 0;
    w.l1 = a.u_l1;
    w.off = (long long)j << a.u_logn;
    w.scratch = w.off;
    return w;
}

__device__ __forceinline__ void issue(const FsqArgs& a, const Work& w, float2* st, uint64_t pol) {
    if (w.kind == FSQ_LINES) {
        load_linear(st, a.in + w.off, w.lines << w.logn, true, pol);
        return;
    }
    const int l1 = w.l1, l2 = w.logn - l1;
    if (w.kind == FSQ_COLS) {
        const int lc = ilog2c(FSQ_POINTS) - l1;
        load_tile(st, a.in + w.off + ((long long)w.index << lc), l1, lc, 1LL << l2, pol);
    } else {
        const int lr = ilog2c(FSQ_POINTS) - l2;
        load_linear(st, a.scratch + w.scratch + ((long long)w.index << (lr + l2)), FSQ_POINTS, true, pol);
    }
}

template <bool INV, bool TILE_OUT = false>
__device__ __forceinline__ void compute(const FsqArgs& a, const Work& w, float2* st) {
    if (w.kind == FSQ_LINES) {
        const float2* tw = a.tabs.line_tw[w.logn - 6];
        const float s = out_scale<INV>(1LL << w.logn, a.adjoint);
        switch (w.logn) {
            case 6: do_lines<64, INV>(st, a.out, w.off, w.lines, tw, s); break;
            case 7: do_lines<128, INV>(st, a.out, w.off, w.lines, tw, s); break;
            case 8: do_lines<256, INV>(st, a.out, w.off, w.lines, tw, s); break;
            case 9: do_lines<512, INV>(st, a.out, w.off, w.lines, tw, s); break;
            case 10: do_lines<1024, INV>(st, a.out, w.off, w.lines, tw, s); break;
            case 11: do_lines<2048, INV>(st, a.out, w.off, w.lines, tw, s); break;
            default: do_lines<4096, INV>(st, a.out, w.off, w.lines, tw, s); break;
        }
        return;
    }
    const int l1 = w.l1, l2 = w.logn - l1;
    float2* mid = a.scratch + w.scratch;
    if (w.kind == FSQ_COLS) {
        const float2* tw = a.tabs.line_tw[l1 - 6];
        const float2* fine = a.tabs.fine[w.logn - 13];
        const float2* coarse = a.tabs.coarse[w.logn - 13];
        const int col0 = w.index << (ilog2c(FSQ_POINTS) - l1);
        switch (l1) {
            case 6: do_cols<64, INV, TILE_OUT>(st, mid, l2, col0, tw, fine, coarse); break;
            case 7: do_cols<128, INV, TILE_OUT>(st, mid, l2, col0, tw, fine, coarse); break;
            case 8: do_cols<256, INV, TILE_OUT>(st, mid, l2, col0, tw, fine, coarse); break;
            case 9: do_cols<512, INV, TILE_OUT>(st, mid, l2, col0, tw, fine, coarse); break;
            default: do_cols<1024, INV, TILE_OUT>(st, mid, l2, col0, tw, fine, coarse); break;
        }
    } else {
        const float2* tw = a.tabs.line_tw[l2 - 6];
        const int row0 = w.index << (ilog2c(FSQ_POINTS) - l2);
        const float2* rows = mid + ((long long)row0 << l2);
        float2* dst = a.out + w.off;
        const float scale = out_scale<INV>(1LL << w.logn, a.adjoint);
        switch (l2) {
            case 7: do_rows<128, INV, TILE_OUT>(st, rows, dst, l1, row0, tw, scale); break;
            case 8: do_rows<256, INV, TILE_OUT>(st, rows, dst, l1, row0, tw, scale); break;
            case 9: do_rows<512, INV, TILE_OUT>(st, rows, dst, l1, row0, tw, scale); break;
            default: do_rows<1024, INV, TILE_OUT>(st, rows, dst, l1, row0, tw, scale); break;
        }
    }
}

// Item p runs on CTA p mod gridDim.x; while one item is transformed in one
// stage buffer, the CTA's next item is copied into the other.
template <bool INV>
__global__ void __launch_bounds__(FSQ_THREADS, FSQ_CTAS_PER_SM) k_fsq(const FsqArgs a) {
    extern __shared__ __align__(128) float2 smem[];
    const uint64_t pol = policy_evict_first();
    int p = blockIdx.x;
    if (p >= a.nitems) return;
    issue(a, get_work(a, p), smem, pol);
    cp_async_commit();
    int s = 0;
    for (; p < a.nitems; p += gridDim.x) {
        const int q = p + gridDim.x;
        if (q < a.nitems) issue(a, get_work(a, q), smem + (s ^ 1) * QSTAGE, pol);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();  // this item's copies have landed for every thread
        compute<INV>(a, get_work(a, p), smem + s * QSTAGE);
        __syncthreads();  // the stage is free before the next item's copies target it
        s ^= 1;
    }
    cp_async_wait<0>();
}


// ---- TMA form of the uniform four-step passes (n = 2^16 .. 2^20) -------------
//
// For these sizes every tile is 4, 8 or 16 columns wide (32-, 64- or 128-byte
// rows), and the chunk-pair swizzle of tidx() is exactly the TMA swizzle of
// that row width (SWIZZLE_32B / 64B / 128B: 16-byte chunk index XOR address
// bits 7..9).  So the tiles move with tensor copies issued by one thread:
// column items load n1/256 boxes of C columns x 256 rows from the input and
// store their finished tile to the intermediate the same way; row items load
// their 4096 contiguous points with one 1-D bulk copy and store the transposed
// tile as boxes of RW columns x 256 rows of the output.  Loads complete on a
// per-stage mbarrier (bounded wait); a stage is refilled only after the bulk
// store that read it has finished reading.

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, const void* src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(smem_u32(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

constexpr int TMA_BOX_ROWS = 256;

// thread 0: item p's data into stage `st`, counted on `bar`
__device__ __forceinline__ void tma_issue(const FsqArgs& a, const FsqMaps& m, const Work& w, float2* st,
                                          uint64_t* bar) {
    const int l1 = w.l1, l2 = w.logn - l1;
    mbar_arrive_expect_tx(bar, FSQ_POINTS * (uint32_t)sizeof(float2));
    const long long j = w.off >> w.logn;  // transform index in this chunk
    if (w.kind == FSQ_COLS) {
        const int lc = ilog2c(FSQ_POINTS) - l1;
        const int x = (w.index << lc) * 2;  // floats
        const int C = 1 << lc;
        for (int k = 0; k < (1 << l1) / TMA_BOX_ROWS; ++k)
            tma_load_2d(st + k * TMA_BOX_ROWS * C, &m.ld, x, (int)(j << l1) + k * TMA_BOX_ROWS, bar);
    } else {
        const int lr = ilog2c(FSQ_POINTS) - l2;
        bulk_g2s(st, a.scratch + w.scratch + ((long long)w.index << (lr + l2)), FSQ_POINTS * (uint32_t)sizeof(float2),
                 bar);
    }
}

// thread 0: the finished tile of item w from stage `st`
__device__ __forceinline__ void tma_store(const FsqMaps& m, const Work& w, const float2* st) {
    const int l1 = w.l1, l2 = w.logn - l1;
    const long long j = w.off >> w.logn;
    if (w.kind == FSQ_COLS) {
        const int lc = ilog2c(FSQ_POINTS) - l1, C = 1 << lc;
        const int x = (w.index << lc) * 2;
        for (int k = 0; k < (1 << l1) / TMA_BOX_ROWS; ++k)
            tma_store_2d(&m.st, x, (int)(j << l1) + k * TMA_BOX_ROWS, st + k * TMA_BOX_ROWS * C);
    } else {
        const int lr = ilog2c(FSQ_POINTS) - l2, RW = 1 << lr;
        const int x = (w.index << lr) * 2;  // first row of the group = first output column
        for (int k = 0; k < (1 << l2) / TMA_BOX_ROWS; ++k)
            tma_store_2d(&m.st, x, (int)(j << l2) + k * TMA_BOX_ROWS, st + k * TMA_BOX_ROWS * RW);
    }
    bulk_commit();
}

template <bool INV>
__global__ void __launch_bounds__(FSQ_THREADS, FSQ_CTAS_PER_SM)
    k_fsq_tma(const __grid_constant__ FsqArgs a, const __grid_constant__ FsqMaps m, int* dev_err) {
    extern __shared__ __align__(1024) unsigned char fsq_raw[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int abort_sh;
    // swizzled tiles need 1024-byte aligned stages (the stage size is 34 KiB)
    float2* smem = reinterpret_cast<float2*>(fsq_raw + ((1024u - (smem_u32(fsq_raw) & 1023u)) & 1023u));
    int p = blockIdx.x;
    if (p >= a.nitems) return;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        abort_sh = 0;
        fence_proxy_async_smem();
        tma_issue(a, m, get_work(a, p), smem, &bar[0]);
    }
    __syncthreads();
    int s = 0;
    uint32_t ph[2] = {0u, 0u};
    for (; p < a.nitems; p += gridDim.x) {
        const int q = p + gridDim.x;
        if (threadIdx.x == 0 && q < a.nitems) {
            bulk_wait_read_all();  // the store that last read stage s^1 has read it
            tma_issue(a, m, get_work(a, q), smem + (s ^ 1) * QSTAGE, &bar[s ^ 1]);
        }
        if (!mbar_wait(&bar[s], ph[s])) abort_sh = 1;
        ph[s] ^= 1u;
        __syncthreads();
        if (abort_sh) break;
        const Work w = get_work(a, p);
        compute<INV, true>(a, w, smem + s * QSTAGE);
        fence_proxy_async_smem();  // the tile's generic writes before the bulk store reads them
        __syncthreads();
        if (threadIdx.x == 0) tma_store(m, w, smem + s * QSTAGE);
        s ^= 1;
    }
    if (threadIdx.x == 0) {
        if (abort_sh) {
            report_device_error(dev_err, DEV_ERR_TMA_TIMEOUT);
            // copies still in flight land before the CTA's shared memory goes away
            mbar_wait(&bar[0], ph[0]);
            mbar_wait(&bar[1], ph[1]);
        }
        bulk_wait_all();
    }
}

// ---- one launch over the device-side descriptor queue -------------------------

// the calling thread's earlier cp.async copies arrive on `bar` when they land
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// An item with its transform's offsets, read from the queue one ticket ahead
// (a 48-byte cp.async into shared memory) and handed to every thread there.
typedef FsqItem QDesc;

__device__ __forceinline__ Work q_work(const QDesc& d) {
    Work w;
    w.kind = d.kind;
    w.logn = d.logn;
    w.index = d.index;
    w.lines = d.lines;
    w.l1 = d.l1;
    w.off = d.kind == FSQ_LINES ? d.off : d.xoff;
    w.scratch = d.kind == FSQ_LINES ? 0 : d.xscratch;
    return w;
}

// thread 0: queue entry p -> dst (shared memory), as one cp.async group
__device__ __forceinline__ void q_prefetch_desc(const FsqQueueArgs& q, int p, QDesc* dst) {
    const float2* src = reinterpret_cast<const float2*>(q.a.items + p);
    float2* d = reinterpret_cast<float2*>(dst);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(QDesc) / 16); ++k) cp_async16(d + 2 * k, src + 2 * k);
    cp_async_commit();
}

// transform index of a TMA item inside its group
__device__ __forceinline__ long long q_group_index(const FsqQueueArgs& q, const QDesc& d) {
    return (d.xoff - q.groups[d.grp].off) >> d.logn;
}

// every thread: item `p`'s data into stage `st`, completion on `bar`
// (256 arrivals: cp.async copies of every thread, or thread 0's bulk copies
// counted in bytes plus 255 plain arrivals)
__device__ __forceinline__ void q_issue(const FsqQueueArgs& q, const QDesc& d, float2* st, uint64_t* bar,
                                        uint64_t pol) {
    const FsqItem& it = d;
    if (it.grp < 0) {
        issue(q.a, q_work(d), st, pol);
        cp_async_mbar_arrive(bar);
        return;
    }
    if (threadIdx.x != 0) {
        mbar_arrive(bar);
        return;
    }
    const FsqGroupMaps& m = q.maps[it.grp];
    const int l1 = it.l1, l2 = it.logn - l1;
    mbar_arrive_expect_tx(bar, FSQ_POINTS * (uint32_t)sizeof(float2));
    const long long j = q_group_index(q, d);
    if (it.kind == FSQ_COLS) {
        const int lc = ilog2c(FSQ_POINTS) - l1;
        const int x = (it.index << lc) * 2;  // floats
        const int C = 1 << lc;
        for (int k = 0; k < (1 << l1) / TMA_BOX_ROWS; ++k)
            tma_load_2d(st + k * TMA_BOX_ROWS * C, &m.ld, x, (int)(j << l1) + k * TMA_BOX_ROWS, bar);
    } else {
        // the intermediate was written by other CTAs (generic and async proxies)
        fence_proxy_async_global();
        const int lr = ilog2c(FSQ_POINTS) - l2;
        bulk_g2s(st, q.a.scratch + d.xscratch + ((long long)it.index << (lr + l2)),
                 FSQ_POINTS * (uint32_t)sizeof(float2), bar);
    }
}

// thread 0: the finished tile of TMA item `it` from stage `st`
__device__ __forceinline__ void q_tma_store(const FsqQueueArgs& q, const QDesc& d, const float2* st) {
    const FsqItem& it = d;
    const FsqGroupMaps& m = q.maps[it.grp];
    const int l1 = it.l1, l2 = it.logn - l1;
    const long long j = q_group_index(q, d);
    if (it.kind == FSQ_COLS) {
        const int lc = ilog2c(FSQ_POINTS) - l1, C = 1 << lc;
        const int x = (it.index << lc) * 2;
        for (int k = 0; k < (1 << l1) / TMA_BOX_ROWS; ++k)
            tma_store_2d(&m.stc, x, (int)(j << l1) + k * TMA_BOX_ROWS, st + k * TMA_BOX_ROWS * C);
    } else {
        const int lr = ilog2c(FSQ_POINTS) - l2, RW = 1 << lr;
        const int x = (it.index << lr) * 2;
        for (int k = 0; k < (1 << l2) / TMA_BOX_ROWS; ++k)
            tma_store_2d(&m.str, x, (int)(j << l2) + k * TMA_BOX_ROWS, st + k * TMA_BOX_ROWS * RW);
    }
    bulk_commit();
}

// COLS items of a transform, counted when each is done
__device__ __forceinline__ int q_cols_needed(int logn) { return fsq_cols_items_dev(logn); }

// thread 0: for a ROWS item, waits (bounded) until every COLS item of its
// transform is counted done; other items need nothing
__device__ __forceinline__ bool q_wait_cols(const FsqQueueArgs& q, const QDesc& it) {
    if (it.kind != FSQ_ROWS) return true;
    const int need = q_cols_needed(it.logn);
    if (ld_acquire_gpu(q.counters + 1 + it.xform) >= need) return true;
    const uint64_t t0 = globaltimer_ns();
    while (ld_acquire_gpu(q.counters + 1 + it.xform) < need)
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) return false;
    return true;
}

__device__ __forceinline__ void red_relaxed_add(int* p, int v) {
    asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void bulk_wait_all_but_one() { asm volatile("cp.async.bulk.wait_group 1;" ::: "memory"); }

// A finished item as thread 0 remembers it until it is counted: x = its
// transform when it is a COLS item (-1 otherwise), tma = it committed a bulk
// store group (TMA items do).
struct QDone {
    int x;
    bool tma;
};

// Finished COLS items thread 0 has not counted yet: their transforms x[0..n),
// tma = one of them committed a bulk store.  A GPU-scope release costs thread 0
// an L2 round trip (~2000 clocks, measured) while the CTA waits for it at the
// next barrier, so up to Q_BATCH items share one.
constexpr int Q_BATCH = 8;
constexpr int Q_HOLD = Q_BATCH + 2;  // the loop counts at Q_BATCH; a wait or the end adds up to two first
// in shared memory, used by thread 0 only (no registers held across the loop)
struct QPend {
    int x[Q_HOLD];
    int n;
    int tma;
};

// thread 0: remember finished item d (a COLS item) for the next count
__device__ __forceinline__ void q_hold(QPend& p, const QDone& d) {
    if (d.x < 0) return;
    p.x[p.n++] = d.x;
    p.tma |= d.tma ? 1 : 0;
}

// thread 0: count the held COLS items; `newer` = a bulk group committed after
// theirs may still be pending.  One release for all of them (an acq_rel fence,
// then relaxed reductions): their tile stores (made by every thread before a
// CTA barrier thread 0 has passed, or by bulk stores, waited for here) are
// visible GPU-wide before ROWS items acquire the counts.
__device__ __forceinline__ void q_count(const FsqQueueArgs& q, QPend& p, bool newer) {
    if (p.n == 0) return;
    if (p.tma) {
        if (newer) bulk_wait_all_but_one();
        else bulk_wait_all();
        fence_proxy_async_global();
    }
    fence_acq_rel_gpu();
#pragma unroll
    for (int k = 0; k < p.n; ++k) red_relaxed_add(q.counters + 1 + p.x[k], 1);
    p.n = 0;
    p.tma = 0;
}

// Tickets are drawn one item ahead (the atomic's latency hides behind an
// item's work), and a finished COLS item is counted at least two items later,
// when its stores have long landed, so no thread stalls on either in steady
// state; up to Q_BATCH of them are counted together, and everything held is
// counted as soon as a CTA finishes an item that is not a COLS item.
// A CTA counts everything it holds before it waits for a ROWS item's
// columns, so no wait depends on its own work.
template <bool INV>
__global__ void __launch_bounds__(FSQ_THREADS, FSQ_CTAS_PER_SM)
    k_fsq_queue(const __grid_constant__ FsqQueueArgs q, int* dev_err) {
    extern __shared__ __align__(1024) unsigned char fsq_raw[];
    __shared__ __align__(8) uint64_t bar[2];
    // descriptor ring: the item of iteration j in slot j % 4 from the time it is
    // drawn (two tickets ahead) until it is done, so that no descriptor is
    // copied (a shared-memory access of thread 0 costs hundreds of clocks while
    // the rest of the CTA waits for it at the next barrier)
    __shared__ QDesc sh_q[4];
    __shared__ int sh_next, sh_ready;
    __shared__ QPend held;  // thread 0: finished COLS items not counted yet
    float2* smem = reinterpret_cast<float2*>(fsq_raw + ((1024u - (smem_u32(fsq_raw) & 1023u)) & 1023u));
    const int n = q.a.nitems;
    const uint64_t pol = policy_evict_first();
    // every item, the first included, is drawn by ticket: a CTA that draws a
    // ROWS item knows that running CTAs hold all of its transform's COLS items
    // Thread 0 works three tickets ahead of the item it issues: t1 (its
    // descriptor in shared memory, its readiness read one iteration ago), t2
    // (descriptor landed this iteration, readiness read now), t3 (the atomic
    // draw, consumed next iteration).  A ROWS item is issued once an acquire
    // load of its transform's column count finds it complete (one load, no
    // fence), and waited for only when that load falls short.
    bool first_ok = true;
    int t1 = n, t2 = n, t3 = n;
    bool rows1 = false;  // thread 0: t1 is a ROWS item
    if (threadIdx.x == 0) {
        held.n = 0;
        held.tma = 0;
        mbar_init(&bar[0], FSQ_THREADS);
        mbar_init(&bar[1], FSQ_THREADS);
        fence_proxy_async_smem();
        const int c = atomicAdd(q.counters, 1);
        sh_next = c;
        if (c < n) {
            const QDesc dc = q.a.items[c];
            t1 = atomicAdd(q.counters, 1);
            if (t1 < n) {
                t2 = atomicAdd(q.counters, 1);
                if (t2 < n) t3 = atomicAdd(q.counters, 1);
                const QDesc d1v = q.a.items[t1];
                sh_q[1] = d1v;
                rows1 = d1v.kind == FSQ_ROWS;
            }
            sh_q[0] = dc;
            first_ok = q_wait_cols(q, dc);
        }
        if (t2 < n) q_prefetch_desc(q, t2, &sh_q[2]);
        else cp_async_commit();
    }
    if (__syncthreads_or(!first_ok)) {
        if (threadIdx.x == 0) report_device_error(dev_err, DEV_ERR_QUEUE_TIMEOUT);
        return;
    }
    if (sh_next >= n) return;
    q_issue(q, sh_q[0], smem, &bar[0], pol);
    if (threadIdx.x == 0) cp_async_commit();  // thread 0's groups: descriptor, data, descriptor, ...
    uint32_t ph[2] = {0u, 0u};
    QDone d1{-1, false}, d2{-1, false};  // thread 0: the previous item, the one before it
    bool failed = false;
    for (int j = 0;; ++j) {  // iteration j computes the item of slot j % 4 in stage s = j % 2
        const int s = j & 1;
        if (threadIdx.x == 0) {
            q_hold(held, d2);
            if (held.n >= Q_BATCH || (held.n > 0 && d1.x < 0)) q_count(q, held, d1.tma);
            d2 = d1;
            d1 = QDone{-1, false};
            cp_async_wait<1>();  // t2's descriptor (all but the latest group, the data copies)
            const int nx = t1;   // the item of iteration j + 1
            int ready = 1;
            if (nx < n && rows1) {
                // the acquire orders its columns' stores before this CTA's reads
                const QDesc& dx = sh_q[(j + 1) & 3];
                ready = ld_acquire_gpu(q.counters + 1 + dx.xform) >= q_cols_needed(dx.logn);
            }
            // shift the look-ahead: t2 -> t1, t3 -> t2 (prefetch its descriptor)
            t1 = t2;
            rows1 = false;
            if (t1 < n) {
                const QDesc& dn = sh_q[(j + 2) & 3];
                rows1 = dn.kind == FSQ_ROWS;
            }
            t2 = t3;
            if (t2 < n) {
                t3 = atomicAdd(q.counters, 1);
                q_prefetch_desc(q, t2, &sh_q[(j + 3) & 3]);  // the slot of iteration j - 1, done
            } else {
                cp_async_commit();
            }
            bulk_wait_read_all();  // the other stage is no longer read by a bulk store
            sh_next = nx;
            sh_ready = ready;
        }
        __syncthreads();
        const int nx = sh_next;
        const bool ready = sh_ready != 0;
        if (nx < n && ready) q_issue(q, sh_q[(j + 1) & 3], smem + (s ^ 1) * QSTAGE, &bar[s ^ 1], pol);
        if (threadIdx.x == 0 && (ready || nx >= n)) cp_async_commit();
        const bool landed = mbar_wait(&bar[s], ph[s]);
        ph[s] ^= 1u;
        if (__syncthreads_or(!landed)) {
            failed = true;
            break;
        }
        const QDesc& dc = sh_q[j & 3];
        const Work w = q_work(dc);
        float2* st = smem + s * QSTAGE;
        if (dc.grp >= 0) {
            compute<INV, true>(q.a, w, st);
            fence_proxy_async_smem();  // the tile's generic writes before the bulk store reads them
            __syncthreads();
            if (threadIdx.x == 0) q_tma_store(q, dc, st);
        } else {
            compute<INV>(q.a, w, st);
        }
        if (threadIdx.x == 0) d1 = QDone{dc.kind == FSQ_COLS ? dc.xform : -1, dc.grp >= 0};
        if (nx < n && !ready) {
            // a ROWS item whose columns are still in flight elsewhere: count
            // this CTA's own items first, then wait (bounded)
            __syncthreads();  // every thread's tile stores precede the counts
            bool ok = true;
            if (threadIdx.x == 0) {
                q_hold(held, d2);
                q_hold(held, d1);
                q_count(q, held, false);
                d1 = d2 = QDone{-1, false};
                ok = q_wait_cols(q, sh_q[(j + 1) & 3]);
            }
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            q_issue(q, sh_q[(j + 1) & 3], smem + (s ^ 1) * QSTAGE, &bar[s ^ 1], pol);
            if (threadIdx.x == 0) cp_async_commit();
        }
        __syncthreads();  // every read of stage s (and of its descriptor) is done before either is refilled
        if (nx >= n) break;
    }
    if (threadIdx.x == 0) {
        if (failed) {
            report_device_error(dev_err, DEV_ERR_QUEUE_TIMEOUT);
            // copies still in flight land before the CTA's shared memory goes away
            mbar_wait(&bar[0], ph[0]);
            mbar_wait(&bar[1], ph[1]);
        } else {
            q_hold(held, d2);
            q_hold(held, d1);
            q_count(q, held, false);
        }
        bulk_wait_all();
    }
}

}  // namespace

cudaError_t fsq_launch_queue(const FsqQueueArgs& q, bool inverse, int sms, int* dev_err, cudaStream_t s) {
    if (q.a.nitems <= 0) return cudaSuccess;
    long long grid = (long long)sms * FSQ_CTAS_PER_SM;
    if (grid > q.a.nitems) grid = q.a.nitems;
    if (inverse) k_fsq_queue<true><<<(unsigned)grid, FSQ_THREADS, QSMEM + 1024, s>>>(q, dev_err);
    else k_fsq_queue<false><<<(unsigned)grid, FSQ_THREADS, QSMEM + 1024, s>>>(q, dev_err);
    return cudaGetLastError();
}

cudaError_t fsq_prepare() {
    for (auto k : {k_fsq<false>, k_fsq<true>}) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, QSMEM);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
    }
    for (auto k : {k_fsq_queue<false>, k_fsq_queue<true>}) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, QSMEM + 1024);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
    }
    for (auto k : {k_fsq_tma<false>, k_fsq_tma<true>}) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, QSMEM + 1024);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t fsq_launch(const FsqArgs& a, bool inverse, int sms, cudaStream_t s) {
    if (a.nitems <= 0) return cudaSuccess;
    long long grid = (long long)sms * FSQ_CTAS_PER_SM;
    if (grid > a.nitems) grid = a.nitems;
    if (inverse) k_fsq<true><<<(unsigned)grid, FSQ_THREADS, QSMEM, s>>>(a);
    else k_fsq<false><<<(unsigned)grid, FSQ_THREADS, QSMEM, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fsq_launch_tma(const FsqArgs& a, const FsqMaps& m, bool inverse, int sms, int* dev_err, cudaStream_t s) {
    if (a.nitems <= 0) return cudaSuccess;
    long long grid = (long long)sms * FSQ_CTAS_PER_SM;
    if (grid > a.nitems) grid = a.nitems;
    if (inverse) k_fsq_tma<true><<<(unsigned)grid, FSQ_THREADS, QSMEM + 1024, s>>>(a, m, dev_err);
    else k_fsq_tma<false><<<(unsigned)grid, FSQ_THREADS, QSMEM + 1024, s>>>(a, m, dev_err);
    return cudaGetLastError();
}

}  // namespace mfft
