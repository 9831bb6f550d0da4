// tc_fft.cu -- N = 4096 C2C FFT as two DFT-64 matrix products on the
// Blackwell tensor cores (tcgen05, accumulators in TMEM).
//
// B200 form of the reference's DFT-as-matmul kernel fft_4096_ct_mma
// (src/fft_4096_ct_mma.metal:88-206), which runs radix-8 CT-DIF stages as
// 8x8 FP32 simdgroup matrix products.  Here N = 64 x 64 (x[64*n1 + n2],
// X[k1 + 64*k2]):
//
//   stage 1  Y[k1][n2] = sum_n1 W64^(n1 k1) x[64 n1 + n2]      tensor cores
//   twiddle  Z[n2][k1] = Y[k1][n2] * W4096^(n2 k1)            FP32 CUDA cores
//   stage 2  X[k1 + 64 k2] = sum_n2 W64^(n2 k2) Z[n2][k1]      tensor cores
//
// Each product is D (128 x 64, FP32 in TMEM) = G (128 x 128) * B (128 x 64):
// G is the realified DFT-64 matrix, row 16 (k / 8) + 8 b + k % 8 = component
// b (re/im) of output k (so the two components of an output sit 8 TMEM lanes
// apart, where one thread of a 16-lane TMEM load receives both), column 2n+a
// = component a of input n; B holds one line's data with the
// same interleaved re/im index along K.  G is the A operand, K-major, held in
// tensor memory for the whole kernel (lane m = row m, two 16-bit K values per
// 32-bit column); the line is the B operand in shared memory: MN-major for
// stage 1 (straight from the input layout), K-major for stage 2 (written by
// the stage-1 epilogue).
//
// Precision variants:
//   FP16 split: every operand v is stored as hi = fp16(v), lo = fp16(v - hi)
//               and D = Ghi*Bhi + Ghi*Blo + Glo*Bhi (three products, FP32
//               accumulate), ~22-bit operands.  Lines are scaled by a power
//               of two so |max| = 2^14 (G by 16) to keep lo parts normal;
//               scales are undone exactly in the epilogues.
//   BF16:       one product of bf16 operands.
//
// One persistent CTA per SM, warp-specialised, every hand-off an mbarrier.
// Lines go in pairs: one MMA of N = 128 covers both lines of a pair (the
// tensor core's cost per instruction, not its FLOP rate, bounds N = 64).
//   converter warps 0-7   two groups of four, group g converts line g of each
//                         pair: coalesced 16-byte streaming loads (the pair
//                         two ahead prefetched into L2), the line's power-of-
//                         two scale, its stage-1 operand (hi/lo) into one of
//                         three 64 KB pair buffers
//   MMA warp 16 (1 thread) stage-1 products of a pair, or stage-2 products of
//                         an earlier pair, whichever has its operands first;
//                         the DFT-64 operand G lives in tensor
//                         memory (the A operand), so the tensor core reads
//                         only the operands from shared memory
//   epilogue-1 warps 8-11 stage-1 accumulators (TMEM) -> re/im pairs -> times
//                         W4096^(n2 k1) 2^-10 (one table, the scale change
//                         between the stages folded in) -> stage-2 operands in
//                         the same pair buffer
//   epilogue-2 warps 12-15 stage-2 accumulators -> unscaled X in a shared-
//                         memory tile per line (128-byte swizzle) inside the
//                         pair's own buffer (its operands have been consumed
//                         once the stage-2 products complete), written out by
//                         TMA tensor stores: four boxes of 16 columns x 64
//                         rows; the buffer goes back to the converters once
//                         the stores have read it
// Three TMEM accumulator slots of 128 columns (G in columns 0-127); the
// stage-1 and stage-2 accumulators of a pair share one slot, since the stage-2
// operands exist only after the stage-1 accumulators have been read.  Every
// wait is bounded by the global timer; a wait that gives up sets a CTA-wide
// abort flag, each warp group leaves its loop together (barrier with an OR),
// the MMA thread waits (bounded) for its MMAs, and the CTA frees its TMEM.
#include "capi_internal.h"
#include "fft_common.cuh"
#include "tcgen05.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace mfft {

namespace {

constexpr int TC_N = 4096;
constexpr int TC_R = 64;
constexpr float TC_GSCALE = 16.0f;  // FP16 split: G stored as 16 * DFT-64
constexpr int TC_LINE_EXP = 14;     // FP16 split: line scaled so |max| < 2^14

// Operand layouts: 128-byte swizzle (1024-byte atoms of 8 rows x 128 bytes,
// 16-byte chunk c of row r stored at chunk c ^ (r % 8)), so that the eight
// threads of a quarter-warp storing one 128-byte row hit distinct banks.
//  B1 (B, MN-major): rows = K (128), N = n2 (64 = one 128-byte row per line)
//  B2 (B, K-major):  rows n = k1 (64 per line), K = 2*n2+a (128) = 2 atoms of 64
constexpr uint32_t ATOM_SBO = 1024;   // stride of 8-row groups

__host__ __device__ constexpr uint32_t sw128(uint32_t row, uint32_t chunk) {
    return (row / 8) * 1024 + (row % 8) * 128 + ((chunk ^ (row % 8)) * 16);
}
// K-major operand with `rows` rows: element (row, kk)
__host__ __device__ constexpr uint32_t kmaj_off(uint32_t row, uint32_t kk, uint32_t katom) {
    return (kk / 64) * katom + sw128(row, (kk % 64) / 8) + (kk % 8) * 2;
}
// MN-major B1: element (nn, kk)
__host__ __device__ constexpr uint32_t mnmaj_off(uint32_t nn, uint32_t kk) {
    return sw128(kk, nn / 8) + (nn % 8) * 2;
}

// Tables (FP64 sincospi): G = realified DFT-64 as plain row-major 16-bit
// planes (row m = 16 (k / 8) + 8 b + k % 8, column kk = 2n+a; FP16 hi and lo of 16 * G, and
// BF16 of G) -- the image each lane stores into tensor memory -- and
// T[m] = W4096^m.
__global__ void k_tc_tables(__half* g_hi, __half* g_lo, __nv_bfloat16* g_bf, float2* tw) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // 0 .. 128*128-1
    if (idx < 128 * 128) {
        const int m = idx / 128, kk = idx % 128;
        const int k = 8 * (m >> 4) + (m & 7), b = (m >> 3) & 1, n = kk >> 1, a = kk & 1;
        double s, c;
        sincospi(-2.0 * (double)((n * k) % TC_R) / (double)TC_R, &s, &c);  // W64^(nk) = c + i s
        // out re = c*xr - s*xi ; out im = s*xr + c*xi
        const double gv = (b == 0) ? (a == 0 ? c : -s) : (a == 0 ? s : c);
        const float gs = (float)(gv * TC_GSCALE);
        const __half h = __float2half_rn(gs);
        g_hi[idx] = h;
        g_lo[idx] = __float2half_rn(gs - __half2float(h));
        g_bf[idx] = __float2bfloat16_rn((float)gv);
    }
    if (idx < TC_N) {
        double s, c;
        sincospi(-2.0 * (double)idx / (double)TC_N, &s, &c);
        tw[idx] = make_float2((float)c, (float)s);
    }
}

// power of two s with max*s < 2^TC_LINE_EXP (1 for max == 0)
__device__ __forceinline__ float line_scale(float mx) {
    if (!(mx > 0.f)) return 1.f;
    int e;
    frexpf(mx, &e);  // mx = f * 2^e, f in [0.5, 1)
    return ldexpf(1.f, TC_LINE_EXP - e);
}

__device__ __forceinline__ void tma_store_2d_tc(const CUtensorMap* map, int x, int y, const void* src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(smem_u32(src))
                 : "memory");
}

// bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned) into L2
__device__ __forceinline__ void prefetch_l2(const void* g, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(g), "r"(bytes) : "memory");
}

// ---- the warp-specialised kernel --------------------------------------------
//
// Lines go through in pairs: one MMA of N = 128 covers both lines of a pair,
// so a line costs 24 MMA instructions (split) instead of 48, and the tensor
// core's per-instruction cost is paid once per two lines.
constexpr int TW_CONV = 0, TW_EPI1 = 8, TW_EPI2 = 12, TW_MMA = 16;  // first warp of each role
constexpr int TW_THREADS = 17 * 32;
// pair buffers: the stage-1 operands, then the stage-2 operands, then the two
// lines' output tiles of the same pair
constexpr int TW_NOP = 3;
constexpr int TW_NSLOT = 3;  // TMEM accumulator slots of 128 columns; D1 and D2 of a pair share one
constexpr int TW_PF = 2;     // L2 prefetch distance of the converters, in pairs
constexpr int TW_NS1 = 8;    // line-scale ring, in pairs (the converters run at most 3 pairs ahead of epilogue 2)
constexpr uint32_t TW_OPB = 65536;                       // one pair buffer: hi 32 KB + lo 32 KB
constexpr uint32_t TW_LO = 32768;                        // lo plane offset inside a pair buffer
constexpr uint32_t TW_TAB = TW_NOP * TW_OPB;             // twiddle table: 4096 float2 = 32 KB
constexpr uint32_t TW_SMEM = TW_TAB + 32768 + 1024;      // + alignment slack
constexpr long long TW_MAX_LINES = 1LL << 24;            // per launch: output row 64*line fits in 31 bits
constexpr uint32_t TW_GCOL = 0, TW_DCOL = 128;           // TMEM columns: G, then the slots
// named barriers (0 is __syncthreads): converter group g uses 1 + g; 5 joins the
// epilogue and MMA warps once the table and G are set up
constexpr int TW_BAR_CONV = 1, TW_BAR_EPI1 = 3, TW_BAR_EPI2 = 4, TW_BAR_SETUP = 5;
// pair operand layouts (bytes inside a plane): B1 MN-major, line g's 128 K
// rows of 128 bytes at g * 16 KB (the MMA's second 64-column N group at LBO =
// 16 KB); B2 K-major, 128 rows (line g's k1 at row 64 g + k1), K atoms of 64
// at 16 KB
constexpr uint32_t B1_LINE = 16384;
constexpr uint32_t B2P_KATOM = 16384;

// bounded wait that also leaves when another role has aborted the CTA
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort) return false;
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
            *abort = 1;
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void named_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// 2 FP32 values -> 4 bytes of the operand (hi/lo planes at b and b + lo, or bf16)
template <bool SPLIT>
__device__ __forceinline__ void store_pair_p(uint8_t* b, uint32_t lo, uint32_t off, float x0, float x1) {
    if constexpr (SPLIT) {
        const __half2 h = __floats2half2_rn(x0, x1);
        const float2 hf = __half22float2(h);
        const __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
        *reinterpret_cast<__half2*>(b + off) = h;
        *reinterpret_cast<__half2*>(b + lo + off) = l;
    } else {
        *reinterpret_cast<__nv_bfloat162*>(b + off) = __floats2bfloat162_rn(x0, x1);
    }
}

// Column orders of the two products (the N index of each MMA), chosen so that
// every shared-memory access of the converters and the epilogues is free of
// bank conflicts for the 16-lane TMEM load layout:
//   stage 1: column j = 8 r + 2 c + s holds n2 = s + 2 r0 + 4 r1 + 8 c + 32 r2
//            (r = r2 r1 r0 in bits), so a lane's steps 2 rp, 2 rp + 1 cover four
//            consecutive n2, one 16-byte chunk of the stage-2 operand;
//   stage 2: output k1 sits in column stage2_col(k1) (bits 1, 2, 3 of k1 moved
//            to 3, 1, 2), so that column j = 8 r + 2 c + s holds
//            k1 = 16 (r / 2) + 4 c + 2 (r % 2) + s.
__host__ __device__ constexpr int stage1_col(int n2) {  // inverse of the stage-1 order, n2 -> column
    return (n2 & 1) | (((n2 >> 3) & 3) << 1) | (((n2 >> 1) & 1) << 3) | (((n2 >> 2) & 1) << 4) | (((n2 >> 5) & 1) << 5);
}
__host__ __device__ constexpr int stage2_col(int k1) {
    return (k1 & 1) | (((k1 >> 2) & 1) << 1) | (((k1 >> 3) & 1) << 2) | (((k1 >> 1) & 1) << 3) | (k1 & 48);
}

// 8 FP32 values -> one 16-byte chunk of the operand (hi/lo planes at b and b + lo, or bf16)
template <bool SPLIT>
__device__ __forceinline__ void store_chunk_p(uint8_t* b, uint32_t lo, uint32_t off, const float (&x)[8]) {
    if constexpr (SPLIT) {
        uint32_t hi[4], lw[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __half2 h = __floats2half2_rn(x[2 * i], x[2 * i + 1]);
            const float2 hf = __half22float2(h);
            const __half2 l = __floats2half2_rn(x[2 * i] - hf.x, x[2 * i + 1] - hf.y);
            hi[i] = *reinterpret_cast<const uint32_t*>(&h);
            lw[i] = *reinterpret_cast<const uint32_t*>(&l);
        }
        *reinterpret_cast<uint4*>(b + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(b + lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    } else {
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
            w[i] = *reinterpret_cast<const uint32_t*>(&h);
        }
        *reinterpret_cast<uint4*>(b + off) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

template <bool SPLIT, bool INV>
__global__ void __launch_bounds__(TW_THREADS, 1)
    k_fft4096_tcw(const float2* __restrict__ in, long long batch, const __grid_constant__ CUtensorMap omap,
                  const uint4* __restrict__ gplain, const float2* __restrict__ tw, int* dev_err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t op_full1[TW_NOP], op_full2[TW_NOP], op_empty[TW_NOP];
    __shared__ __align__(8) uint64_t d1_full[TW_NSLOT], d2_full[TW_NSLOT], d_empty[TW_NSLOT];
    __shared__ __align__(8) uint64_t s1_full[TW_NS1], drain;
    __shared__ float s1ring[TW_NS1][2];
    __shared__ float red[2][2][4];  // [converter group][pair parity][warp]
    __shared__ uint32_t tmem_base_sh;
    __shared__ int abort_flag;
    volatile int* abort_sh = &abort_flag;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const long long G = gridDim.x;
    const long long npairs = (batch + 1) / 2;
    const long long nloc = npairs > (long long)blockIdx.x ? (npairs - blockIdx.x + G - 1) / G : 0;
    // the first TW_PF pairs into L2 while the CTA sets up
    if (tid < 2 * TW_PF && tid / 2 < nloc && 2 * (blockIdx.x + (tid / 2) * G) + (tid & 1) < batch)
        prefetch_l2(in + (size_t)(2 * (blockIdx.x + (tid / 2) * G) + (tid & 1)) * TC_N, TC_N * sizeof(float2));
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_u32(smem);
    float2* tab = reinterpret_cast<float2*>(smem + TW_TAB);
    constexpr uint32_t FMT = SPLIT ? 0u : 1u;
    constexpr uint32_t IDESC1 = tc::idesc_f16(FMT, 1u, 128, 128);
    constexpr uint32_t IDESC2 = tc::idesc_f16(FMT, 0u, 128, 128);

    if (tid == 0) {
        for (int j = 0; j < TW_NOP; ++j) {
            mbar_init(&op_full1[j], 256);
            mbar_init(&op_full2[j], 128);
            mbar_init(&op_empty[j], 1);
        }
        for (int j = 0; j < TW_NSLOT; ++j) {
            mbar_init(&d1_full[j], 1);
            mbar_init(&d2_full[j], 1);
            mbar_init(&d_empty[j], 128);
        }
        for (int j = 0; j < TW_NS1; ++j) mbar_init(&s1_full[j], 2);
        mbar_init(&drain, 1);
        abort_flag = 0;
        fence_proxy_async_smem();
    }
    if (warp == TW_MMA) {
        tc::tmem_alloc(&tmem_base_sh, 512);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tmem_base_sh;

    // The epilogue and MMA warps set up the twiddle table and G while the
    // converters start on the first pair.
    if (warp >= TW_EPI1) {
        // T[n2*64 + (k1 + 4 * ((n2 >> 3) & 3)) % 64] = W4096^(n2 k1) (times 2^-10
        // for the split: the stage-2 operand is D1 / (16 s1) * W * s1 / 64).  A
        // half-warp of epilogue 1 reads 4 consecutive k1 of the rows n2 = n + 8c,
        // c = 0..3; the rotation puts the four rows on distinct banks.
        if (warp < TW_EPI2 + 4) {
            for (int i = tid - 32 * TW_EPI1; i < TC_N; i += 256) {
                const int n2 = i >> 6, k1 = ((i & 63) - 4 * ((n2 >> 3) & 3)) & 63;
                const float2 w = __ldg(tw + ((n2 * k1) & (TC_N - 1)));
                const float sc = SPLIT ? 0.0009765625f : 1.f;
                tab[i] = make_float2(w.x * sc, w.y * sc);
            }
        }
    }
    // G into tensor memory: lane m holds row m (hi in columns 0-63, lo in 64-127)
    if (warp >= TW_EPI1 && warp < TW_EPI1 + 4) {
        const int m = 32 * (warp & 3) + lane;
        const uint32_t lane_off = (uint32_t)(32 * (warp & 3)) << 16;
#pragma unroll 1
        for (int pl = 0; pl < (SPLIT ? 2 : 1); ++pl) {
            // plane pl: hi (SPLIT) / bf16 at gplain, lo at gplain + 128*128 halves
            const uint4* row = gplain + (size_t)pl * 2048 + (size_t)m * 16;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t r[32];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const uint4 u = __ldg(row + 8 * h + q);
                    r[4 * q] = u.x;
                    r[4 * q + 1] = u.y;
                    r[4 * q + 2] = u.z;
                    r[4 * q + 3] = u.w;
                }
                tc::tmem_st32(tbase + lane_off + TW_GCOL + 64 * pl + 32 * h, r);
            }
        }
    }
    if (warp >= TW_EPI1) {
        tc::fence_before_sync();
        named_sync(TW_BAR_SETUP, 32 * (TW_MMA + 1 - TW_EPI1));
        tc::fence_after_sync();
    }

    if (warp < TW_CONV + 8) {
        // ---------------- converters: group g writes line g of each pair ----------------
        const int g = warp >> 2, wl = warp & 3, ctid = tid & 127;
#pragma unroll 1
        for (long long i = 0; i < nloc; ++i) {
            const long long P = blockIdx.x + i * G;
            const long long f = 2 * P + g;
            const bool valid = f < batch;
            const int o = (int)i % TW_NOP;
            if (ctid == 0 && i + TW_PF < nloc && 2 * (P + TW_PF * G) + g < batch)
                prefetch_l2(in + (size_t)(2 * (P + TW_PF * G) + g) * TC_N, TC_N * sizeof(float2));
            // float4 q = ctid + 128 r holds x[2q], x[2q+1]: n1 = wl + 4 r, n2 = 2 lane (+1)
            float4 cur[16];
            if (valid) {
                const float4* src = reinterpret_cast<const float4*>(in + (size_t)f * TC_N) + ctid;
#pragma unroll
                for (int r = 0; r < 16; ++r) cur[r] = __ldcs(src + 128 * r);
            } else {
#pragma unroll
                for (int r = 0; r < 16; ++r) cur[r] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            if constexpr (INV) {
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    cur[r].y = -cur[r].y;
                    cur[r].w = -cur[r].w;
                }
            }
            if constexpr (SPLIT) {
                float mx = 0.f;
#pragma unroll
                for (int r = 0; r < 16; ++r)
                    mx = fmaxf(mx, fmaxf(fmaxf(fabsf(cur[r].x), fabsf(cur[r].y)), fmaxf(fabsf(cur[r].z), fabsf(cur[r].w))));
#pragma unroll
                for (int sh = 16; sh > 0; sh >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, sh));
                if (lane == 0) red[g][i & 1][wl] = mx;
            }
            // the pair buffer is free once the previous pair's stage-2 products are done
            bool ok = true;
            if (ctid == 0) ok = wait_or_abort(&op_empty[o], (uint32_t)((((int)i / TW_NOP) & 1) ^ 1), abort_sh);
            if (bar_or(TW_BAR_CONV + g, 128, !ok)) break;
            float s1 = 1.f;
            if constexpr (SPLIT)
                s1 = line_scale(fmaxf(fmaxf(red[g][i & 1][0], red[g][i & 1][1]), fmaxf(red[g][i & 1][2], red[g][i & 1][3])));
            uint8_t* bp = smem + (uint32_t)o * TW_OPB + (uint32_t)g * B1_LINE;
            // columns j, j + 1 of the operand take n2 = 2 lane, 2 lane + 1 (the
            // stage-1 column order); a warp writes one 128-byte row per row: no
            // bank conflicts
            const int j0 = stage1_col(2 * lane);
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const int n1 = wl + 4 * r;
                const float4 v = cur[r];
                store_pair_p<SPLIT>(bp, TW_LO, mnmaj_off(j0, 2 * n1), v.x * s1, v.z * s1);
                store_pair_p<SPLIT>(bp, TW_LO, mnmaj_off(j0, 2 * n1 + 1), v.y * s1, v.w * s1);
            }
            if (ctid == 0) {
                s1ring[(int)i % TW_NS1][g] = s1;
                mbar_arrive(&s1_full[(int)i % TW_NS1]);
            }
            fence_proxy_async_smem();  // the operand's generic writes before the tensor core reads them
            mbar_arrive(&op_full1[o]);
        }
    } else if (warp < TW_EPI1 + 4) {
        // ---------------- epilogue 1: twiddle and the stage-2 operands ----------------
        // 16-lane TMEM loads: half hb of the warp's lane quarter q gives lane
        // (rl = lane / 4) the real and imaginary rows of k1 = 16 q + 8 hb + rl,
        // columns j = 8 r + 2 c + s (c = lane % 4, r = 0..7, s = 0, 1), which
        // hold n2 = stage1_n2(j)
        const int q = warp & 3, m = 32 * q + lane, rl = lane >> 2, c = lane & 3;
        const uint32_t lane_q = (uint32_t)(32 * q) << 16;
        const int rot = 4 * c;  // table rotation of this lane's rows n2 (bits 3-4 of n2 = c)
#pragma unroll 1
        for (long long i = 0; i < nloc; ++i) {
            const int sl = (int)i % TW_NSLOT, o = (int)i % TW_NOP;
            bool ok = true;
            if (m == 0) ok = wait_or_abort(&d1_full[sl], (uint32_t)(((int)i / TW_NSLOT) & 1), abort_sh);
            if (bar_or(TW_BAR_EPI1, 128, !ok)) break;
            tc::fence_after_sync();
            uint8_t* bp = smem + (uint32_t)o * TW_OPB;
            // block gh = (line g, lane half hb) = (gh / 2, gh % 2); the load of
            // block gh + 1 is in flight while block gh is processed
            auto taddr = [&](int gh) {
                return tbase + lane_q + ((uint32_t)(16 * (gh & 1)) << 16) + TW_DCOL + 128 * sl + 64 * (gh >> 1);
            };
            auto proc = [&](const uint32_t(&v)[32], int gh) {
                const int k1 = 16 * q + 8 * (gh & 1) + rl;
                const int row = 64 * (gh >> 1) + stage2_col(k1);
                const float2* trow = tab + ((k1 + rot) & 63);
#pragma unroll
                for (int rp = 0; rp < 4; ++rp) {
                    // steps r = 2 rp, 2 rp + 1 hold n2 = nb .. nb + 3: one 16-byte chunk (K = 2 nb .. 2 nb + 7)
                    const int nb = 4 * (rp & 1) + 8 * c + 32 * (rp >> 1);
                    float x[8];
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        const int r = 2 * rp + (t >> 1), sb = t & 1;
                        const float2 z = cmul(make_float2(__uint_as_float(v[4 * r + sb]), __uint_as_float(v[4 * r + 2 + sb])),
                                              trow[(nb + t) * 64]);
                        x[2 * t] = z.x;
                        x[2 * t + 1] = z.y;
                    }
                    store_chunk_p<SPLIT>(bp, TW_LO, kmaj_off(row, 2 * nb, B2P_KATOM), x);
                }
            };
            uint32_t va[32], vb[32];
            tc::tmem_ld16x256_issue(taddr(0), va);
            tc::tmem_wait_ld(va);
            tc::tmem_ld16x256_issue(taddr(1), vb);
            proc(va, 0);
            tc::tmem_wait_ld(vb);
            tc::tmem_ld16x256_issue(taddr(2), va);
            proc(vb, 1);
            tc::tmem_wait_ld(va);
            tc::tmem_ld16x256_issue(taddr(3), vb);
            proc(va, 2);
            tc::tmem_wait_ld(vb);
            proc(vb, 3);
            // D1 has been read (its slot takes this pair's D2) and the operands written
            tc::fence_before_sync();
            fence_proxy_async_smem();
            mbar_arrive(&op_full2[o]);
        }
    } else if (warp < TW_EPI2 + 4) {
        // ---------------- epilogue 2: X out ----------------
        // 16-lane TMEM loads as in epilogue 1: lane (rl, c) gets X[k1 + 64 k2] for
        // k2 = 16 q + 8 hb + rl and the stage-2 column j = 8 r + 2 c + s, which
        // holds k1 = 16 (r / 2) + 4 c + 2 (r % 2) + s.  Tile of line g: bytes
        // [32 KB g, 32 KB (g + 1)) of the pair buffer, box bx (columns k1 = 16 bx
        // .. 16 bx + 15) of 64 rows k2 x 128 bytes, 16-byte chunk ch of row k2 at
        // ch ^ (k2 % 8) (the tensor map's 128-byte swizzle)
        const int q = warp & 3, m = 32 * q + lane, rl = lane >> 2, c = lane & 3;
        const uint32_t lane_q = (uint32_t)(32 * q) << 16;
#pragma unroll 1
        for (long long i = 0; i < nloc; ++i) {
            const long long P = blockIdx.x + i * G;
            const int sl = (int)i % TW_NSLOT, o = (int)i % TW_NOP;
            bool ok = true;
            if (m == 0)
                ok = wait_or_abort(&d2_full[sl], (uint32_t)(((int)i / TW_NSLOT) & 1), abort_sh) &&
                     wait_or_abort(&s1_full[(int)i % TW_NS1], (uint32_t)(((int)i / TW_NS1) & 1), abort_sh);
            if (bar_or(TW_BAR_EPI2, 128, !ok)) break;
            tc::fence_after_sync();
            // the stage-2 products have completed, so the pair buffer takes the
            // two output tiles (line g at g * 32 KB); block gh = (line g, lane half
            // hb) = (gh / 2, gh % 2), the load of block gh + 1 in flight while block
            // gh is processed
            uint8_t* bp = smem + (uint32_t)o * TW_OPB;
            auto taddr = [&](int gh) {
                return tbase + lane_q + ((uint32_t)(16 * (gh & 1)) << 16) + TW_DCOL + 128 * sl + 64 * (gh >> 1);
            };
            // X = D2 / (16 s2), s2 = s1 / 64 (split); X = D2 (bf16)
            const float sc0 = (INV ? 1.f / (float)TC_N : 1.f) * (SPLIT ? 4.f / s1ring[(int)i % TW_NS1][0] : 1.f);
            const float sc1 = (INV ? 1.f / (float)TC_N : 1.f) * (SPLIT ? 4.f / s1ring[(int)i % TW_NS1][1] : 1.f);
            const bool live1 = 2 * P + 1 < batch;  // false for the second line of an odd batch's last pair
            auto proc = [&](const uint32_t(&v)[32], int gh) {
                const int g = gh >> 1;
                const float sc = g ? sc1 : sc0;
                const int k2 = 16 * q + 8 * (gh & 1) + rl;
                uint8_t* rowp = bp + (uint32_t)g * 32768 + (uint32_t)k2 * 128;
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    float4 o4 = make_float4(__uint_as_float(v[4 * r]) * sc, __uint_as_float(v[4 * r + 2]) * sc,
                                            __uint_as_float(v[4 * r + 1]) * sc, __uint_as_float(v[4 * r + 3]) * sc);
                    if constexpr (INV) {
                        o4.y = -o4.y;
                        o4.w = -o4.w;
                    }
                    const int ch = (r & 1) + 2 * c;  // X[k1], X[k1 + 1], k1 = 16 (r / 2) + 4 c + 2 (r % 2)
                    *reinterpret_cast<float4*>(rowp + (uint32_t)(r >> 1) * 8192 + ((ch ^ (k2 & 7)) << 4)) = o4;
                }
            };
            // line g's tile is complete: four tensor stores of its boxes
            auto store_line = [&](int g) {
                fence_proxy_async_smem();  // the tile's generic writes before the tensor stores read it
                named_sync(TW_BAR_EPI2, 128);
                if (m == 0) {
                    const uint8_t* ot = bp + (uint32_t)g * 32768;
#pragma unroll
                    for (int bx = 0; bx < 4; ++bx) tma_store_2d_tc(&omap, 32 * bx, (int)(64 * (2 * P + g)), ot + bx * 8192);
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
            };
            uint32_t va[32], vb[32];
            tc::tmem_ld16x256_issue(taddr(0), va);
            tc::tmem_wait_ld(va);
            tc::tmem_ld16x256_issue(taddr(1), vb);
            proc(va, 0);
            tc::tmem_wait_ld(vb);
            tc::tmem_ld16x256_issue(taddr(2), va);
            proc(vb, 1);
            store_line(0);
            tc::tmem_wait_ld(va);
            tc::tmem_ld16x256_issue(taddr(3), vb);
            if (live1) proc(va, 2);
            tc::tmem_wait_ld(vb);
            tc::fence_before_sync();
            mbar_arrive(&d_empty[sl]);  // the slot may take a later pair
            if (live1) {
                proc(vb, 3);
                store_line(1);
            }
            // the pair buffer goes back to the converters once the tensor stores have read it
            if (m == 0) {
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                mbar_arrive(&op_empty[o]);
            }
        }
        if (m == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    } else if (warp == TW_MMA && lane == 0) {
        // ---------------- MMA issue ----------------
        // Stage 1 of pair i1 and stage 2 of pair i2 < i1, whichever has its
        // operands first (stage 2 first when both do), so that the tensor core
        // runs the ready stage while the other's operands are still being made.
        constexpr int NPROD = SPLIT ? 3 : 1;
        const uint32_t g_hi = tbase + TW_GCOL, g_lo = g_hi + 64;
        bool aborted = false;
        long long i1 = 0, i2 = 0;
        uint64_t t0 = globaltimer_ns();
#pragma unroll 1
        while (i2 < nloc) {
            bool issued = false;
            if (i2 < i1) {
                const int o = (int)i2 % TW_NOP, sl = (int)i2 % TW_NSLOT;
                // the stage-2 operands are written only after epilogue 1 has read D1,
                // so D2 may overwrite it in the same slot
                if (mbar_test_wait(&op_full2[o], (uint32_t)(((int)i2 / TW_NOP) & 1))) {
                    tc::fence_after_sync();
                    const uint32_t bb = sbase + (uint32_t)o * TW_OPB;
                    const uint32_t dd = tbase + TW_DCOL + 128 * sl;
#pragma unroll
                    for (int pr = 0; pr < NPROD; ++pr) {
                        const uint32_t ga = pr == 2 ? g_lo : g_hi;
                        const uint32_t bpl = bb + (pr == 1 ? TW_LO : 0u);
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            tc::mma_f16_ts(dd, ga + 8 * j,
                                           tc::smem_desc(bpl + (j / 4) * B2P_KATOM + (j % 4) * 32, 16, ATOM_SBO,
                                                         tc::LAYOUT_SW128),
                                           IDESC2, (pr > 0 || j > 0) ? 1u : 0u);
                    }
                    tc::mma_commit(&d2_full[sl]);
                    ++i2;
                    issued = true;
                }
            }
            if (!issued && i1 < nloc) {
                const int o = (int)i1 % TW_NOP, sl = (int)i1 % TW_NSLOT;
                if (mbar_test_wait(&op_full1[o], (uint32_t)(((int)i1 / TW_NOP) & 1)) &&
                    mbar_test_wait(&d_empty[sl], (uint32_t)((((int)i1 / TW_NSLOT) & 1) ^ 1))) {
                    tc::fence_after_sync();
                    const uint32_t bb = sbase + (uint32_t)o * TW_OPB;
                    const uint32_t dd = tbase + TW_DCOL + 128 * sl;
#pragma unroll
                    for (int pr = 0; pr < NPROD; ++pr) {
                        const uint32_t ga = pr == 2 ? g_lo : g_hi;
                        const uint32_t bpl = bb + (pr == 1 ? TW_LO : 0u);
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            tc::mma_f16_ts(dd, ga + 8 * j,
                                           tc::smem_desc(bpl + 2 * j * ATOM_SBO, B1_LINE, ATOM_SBO, tc::LAYOUT_SW128),
                                           IDESC1, (pr > 0 || j > 0) ? 1u : 0u);
                    }
                    tc::mma_commit(&d1_full[sl]);
                    ++i1;
                    issued = true;
                }
            }
            if (issued) {
                t0 = globaltimer_ns();
            } else if (*abort_sh || globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
                *abort_sh = 1;
                aborted = true;
                break;
            }
        }
        if (aborted) {
            // every MMA this thread issued completes before the CTA frees its tensor memory
            tc::mma_commit(&drain);
            mbar_wait(&drain, 0);
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0 && abort_flag) report_device_error(dev_err, DEV_ERR_MMA_TIMEOUT);
    if (warp == TW_MMA) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tbase, 512);
    }
}

// Launches over at most TW_MAX_LINES lines each (an even count, so pairs never
// straddle launches); the output goes through a tensor map of the chunk's
// lines as 64-row x 512-byte blocks.
template <bool SPLIT, bool INV>
cudaError_t launch_tcw(const float2* in, float2* out, long long batch, const uint4* gplain, const float2* tw,
                       int* dev_err, int sms, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(k_fft4096_tcw<SPLIT, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TW_SMEM);
    if (e != cudaSuccess) return e;
    for (long long b0 = 0; b0 < batch; b0 += TW_MAX_LINES) {
        const long long nb = batch - b0 < TW_MAX_LINES ? batch - b0 : TW_MAX_LINES;
        CUtensorMap omap;
        if (!encode_rows(&omap, out + b0 * TC_N, (uint64_t)nb * TC_R, TC_R, 16, TC_R)) return cudaErrorInvalidValue;
        const long long pairs = (nb + 1) / 2;
        const long long blocks = pairs < sms ? pairs : sms;
        k_fft4096_tcw<SPLIT, INV><<<(unsigned)blocks, TW_THREADS, TW_SMEM, s>>>(in + b0 * TC_N, nb, omap, gplain, tw,
                                                                                 dev_err);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

// tables: [G hi 32 KB][G lo 32 KB][G bf16 32 KB][T 4096 float2 = 32 KB]
int tc_plan_init(mfft_plan* p) {
    if (p->n != TC_N || p->tc.ready) return MFFT_SUCCESS;
    void* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, 4 * 32768);
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "tensor-core tables: %s", cudaGetErrorString(e));
    uint8_t* b = (uint8_t*)buf;
    k_tc_tables<<<(128 * 128 + 255) / 256, 256, 0, p->ctx->stream>>>(
        (__half*)b, (__half*)(b + 32768), (__nv_bfloat16*)(b + 65536), (float2*)(b + 98304));
    e = cudaStreamSynchronize(p->ctx->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFree(buf);
        return cuda_error(e, "tensor-core tables");
    }
    p->tc.dft_tables = buf;
    p->tc.tw = (float2*)(b + 98304);
    p->tc.ready = true;
    return MFFT_SUCCESS;
}

void tc_plan_release(mfft_plan* p) {
    if (p->tc.dft_tables) cudaFree(p->tc.dft_tables);
    p->tc.dft_tables = nullptr;
    p->tc.ready = false;
}

int tc_launch(mfft_plan* p, const float2* in, float2* out, int64_t batch, int direction, int variant,
              cudaStream_t s) {
    const uint8_t* b = (const uint8_t*)p->tc.dft_tables;
    const uint4* g_split = (const uint4*)b;             // hi then lo, contiguous
    const uint4* g_bf = (const uint4*)(b + 65536);
    const int sms = p->ctx->sms;
    int* err = p->ctx->dev_err;
    cudaError_t e;
    const bool inv = (direction == MFFT_INVERSE);
    if (variant == MFFT_TC_FP16_SPLIT3)
        e = inv ? launch_tcw<true, true>(in, out, batch, g_split, p->tc.tw, err, sms, s)
                : launch_tcw<true, false>(in, out, batch, g_split, p->tc.tw, err, sms, s);
    else
        e = inv ? launch_tcw<false, true>(in, out, batch, g_bf, p->tc.tw, err, sms, s)
                : launch_tcw<false, false>(in, out, batch, g_bf, p->tc.tw, err, sms, s);
    if (e != cudaSuccess) return cuda_error(e, "tensor-core FFT launch");
    return MFFT_SUCCESS;
}

}  // namespace mfft

extern "C" int mfft_exec_c2c_tc(mfft_plan* plan, const void* in, void* out, int64_t batch, int direction,
                                int variant, int flags, void* stream) {
    using namespace mfft;
    if (!plan) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "plan is NULL");
    if (plan->n != TC_N)
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, plan->n, -1, -1,
                         "Unsupported FFT size: %lld. The tensor-core path takes n = 4096", (long long)plan->n);
    if (variant != MFFT_TC_FP16_SPLIT3 && variant != MFFT_TC_BF16)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown tensor-core variant %d", variant);
    int st = check_exec_args(in, out, batch, direction, flags);
    if (st) return st;
    if (batch == 0) return MFFT_SUCCESS;
    DeviceGuard g(plan->ctx->device);
    if (!plan->tc.ready) {
        st = tc_plan_init(plan);
        if (st) return st;
    }
    if (flags == MFFT_DEVICE_MEMORY)
        return tc_launch(plan, (const float2*)in, (float2*)out, batch, direction, variant, (cudaStream_t)stream);
    const size_t line = (size_t)TC_N * sizeof(float2);
    return run_host_lines(
        plan->ctx, in, out, batch, line, line,
        [&](const void* di, void* dout, int64_t nl, cudaStream_t s) {
            return tc_launch(plan, (const float2*)di, (float2*)dout, nl, direction, variant, s);
        },
        true);
}
