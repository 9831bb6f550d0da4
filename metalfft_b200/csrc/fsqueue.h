// fsqueue.h -- the persistent item kernel shared by the mixed-size batch
// (multi.cu) and the four-step plans for n > 16384 (fourstep.cu).
//
// Every work item is 4096 complex points handled by one 256-thread CTA (three
// CTAs per SM).  A launch walks its item list with a static schedule (item p
// on CTA p mod grid) and copies the next item's data into the CTA's second
// stage buffer with cp.async while the current item is transformed:
//   LINES  4096/n whole lines of one size n <= 4096
//   COLS   one column tile of a four-step transform n = n1*n2 (n >= 8192):
//          4096/n1 adjacent columns x n1 rows -> column FFTs, times
//          W_n^{col*k1}, into the transform's scratch area (row-major, like
//          the input)
//   ROWS   one row group of that transform: 4096/n2 rows of the scratch
//          area -> row FFTs -> out[k2*n1 + k1] (the transpose folded into a
//          16-byte tile store)
// A four-step batch is two launches on one stream: pass 0 runs every COLS
// (and LINES) item, pass 1 every ROWS item, so no item ever waits for
// another inside a launch and no inter-CTA synchronisation exists.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace mfft {

constexpr int FSQ_THREADS = 256;
constexpr int FSQ_POINTS = 4096;
constexpr int FSQ_CTAS_PER_SM = 3;

enum : int { FSQ_LINES = 0, FSQ_COLS = 1, FSQ_ROWS = 2 };

struct alignas(16) FsqItem {
    int kind;
    int logn;       // log2 of the line size (LINES) or of the transform size
    int index;      // COLS: column tile, ROWS: row group
    int xform;      // four-step transform id (COLS / ROWS)
    long long off;  // LINES: element offset of the first line
    int lines;      // LINES: lines in this item
    int grp;        // queue kernel: TMA group of a COLS / ROWS item (-1: 16-byte copies)
    long long xoff;      // queue kernel, COLS / ROWS: the transform's offset in in / out
    long long xscratch;  //   and of its intermediate (the FsqXform, so one read gives both)
    int l1;              // COLS / ROWS: log2 n1 of the transform's split
    int pad2[3];
};

struct FsqXform {
    long long off;      // element offset of the transform in in / out
    long long scratch;  // element offset of its intermediate in the scratch buffer
    int logn;
    int l1;             // log2 n1 of its split
};

struct FsqTables {
    const float2* line_tw[7];  // line twiddle rows (E = 16) for n = 64 .. 4096
    const float2* fine[8];     // W_n^m = fine[m % 1024] * coarse[m / 1024], n = 2^13 .. 2^20
    const float2* coarse[8];
};

struct FsqArgs {
    const float2* in;
    float2* out;
    float2* scratch;       // four-step intermediates
    const FsqItem* items;  // explicit item list (mixed sizes), or nullptr: uniform pass below
    const FsqXform* xf;
    int nitems;
    // uniform pass over `batch` contiguous four-step transforms of 2^u_logn
    // points: u_kind FSQ_COLS (pass 0) or FSQ_ROWS (pass 1), u_per items each;
    // transform j's intermediate is scratch + j * 2^u_logn
    int u_kind, u_logn, u_per, u_l1;
    // 1: the adjoint of the transform (the inverse unscaled, the forward
    // scaled by 1/n); 0: the transform
    int adjoint;
    FsqTables tabs;
};

// n = 2^m (m >= 13) as n1 * n2: the default n1 = 2^floor(m/2) <= n2, or a
// split n1 = 2^l1 chosen by the autotuner.  The item kernel takes
// 64 <= n1 <= 1024 (column FFTs) and 128 <= n2 <= 1024 (row FFTs); its TMA
// form needs both in {256, 512, 1024} (tiles 16, 8 or 4 columns wide).
inline int fsq_default_l1(int logn) { return logn / 2; }
inline bool fsq_split_ok(int logn, int l1) { return l1 >= 6 && l1 <= 10 && logn - l1 >= 7 && logn - l1 <= 10; }
inline bool fsq_tma_split(int logn, int l1) { return l1 >= 8 && l1 <= 10 && logn - l1 >= 8 && logn - l1 <= 10; }
inline void fsq_split(int logn, int* n1, int* n2, int l1 = -1) {
    if (l1 < 0) l1 = fsq_default_l1(logn);
    *n1 = 1 << l1;
    *n2 = 1 << (logn - l1);
}
// COLS and ROWS items of one four-step transform of 2^logn points: an item
// holds FSQ_POINTS points (FSQ_POINTS / n1 columns of n1, or FSQ_POINTS / n2
// rows of n2), so both passes have n / FSQ_POINTS items whatever the split.
__host__ __device__ inline int fsq_cols_items_dev(int logn) { return (1 << logn) / FSQ_POINTS; }
inline int fsq_cols_items(int logn) { return fsq_cols_items_dev(logn); }
inline int fsq_rows_items(int logn) { return fsq_cols_items_dev(logn); }

// Tensor maps of a uniform pass with TMA tiles: ld = the input viewed as
// rows of n2 points (column pass), st = the column pass's intermediate (rows
// of n2) or the row pass's output (rows of n1, transposed store).  Float
// elements, boxes of (2 x tile width) floats x 256 rows, swizzle of the tile
// row width.
struct FsqMaps {
    CUtensorMap ld;
    CUtensorMap st;
};

// ---- one persistent launch over a device-side descriptor queue -------------
//
// Mixed sizes: every item of a batch (COLS of every four-step transform,
// then LINES, then ROWS) in one array; CTAs draw items by atomic ticket.  A
// ROWS item waits (bounded) until the COLS items of its transform have all
// been counted done; tickets are drawn in array order, so every COLS item is
// held by some CTA before any ROWS item is drawn, and a CTA publishes its
// finished COLS item before it ever waits.  Four-step transforms of one TMA
// size class that sit back to back form a group whose tiles move by TMA.
constexpr int FSQ_MAX_GROUPS = 8;
struct FsqGroup {
    long long off;      // element offset of the group's first transform in in / out
    long long scratch;  // element offset of its first intermediate
    int logn;
    int l1;
};
struct FsqGroupMaps {
    CUtensorMap ld;    // input as rows of n2 (COLS load)
    CUtensorMap stc;   // intermediate as rows of n2 (COLS store)
    CUtensorMap str;   // output as rows of n1 (ROWS store)
};
struct FsqQueueArgs {
    FsqArgs a;        // in, out, scratch, items, xf, nitems, tabs, adjoint
    int* counters;    // [0] next ticket, [1 + x] COLS items done of transform x
    int ngroups;
    FsqGroup groups[FSQ_MAX_GROUPS];
    FsqGroupMaps maps[FSQ_MAX_GROUPS];
};

cudaError_t fsq_prepare();
// Launches one pass over a.nitems items on `s`.
cudaError_t fsq_launch(const FsqArgs& a, bool inverse, int sms, cudaStream_t s);
// The same uniform pass with TMA tiles (four-step n = 2^16 .. 2^20 only).
cudaError_t fsq_launch_tma(const FsqArgs& a, const FsqMaps& m, bool inverse, int sms, int* dev_err, cudaStream_t s);
// The whole queue in one launch; q.counters must be zero when it starts.
cudaError_t fsq_launch_queue(const FsqQueueArgs& q, bool inverse, int sms, int* dev_err, cudaStream_t s);

}  // namespace mfft
