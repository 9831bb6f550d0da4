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
// G is the realified DFT-64 matrix, row 2k+b = component b (re/im) of output
// k, column 2n+a = component a of input n; B holds one line's data with the
// same interleaved re/im index along K.  G is the A operand (K-major, loaded
// into shared memory once per CTA); the line is the B operand: MN-major for
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
// One CTA of 512 threads per SM holds G once and runs four independent
// pipelines of 128 threads, one line each at a time (four lines in flight per
// SM), each with its own B buffers, TMEM columns, commit mbarrier and named
// barrier.  The stage-2 scale is s1/64 (a DFT-64 grows magnitudes by at most
// 64), so no reduction sits between the two products.  A pipeline's first
// thread issues its MMAs and waits on the commit mbarrier with a time limit;
// a timeout sets the device error word and the pipeline leaves its loop; the
// CTA then frees its TMEM and returns.
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

// shared-memory byte offsets from a 1024-byte aligned base (dynamic)
constexpr uint32_t SM_G0 = 0;          // G hi (or bf16) : 128 x 128 halves = 32 KB
constexpr uint32_t SM_G1 = 32768;      // G lo

// Operand layouts: 128-byte swizzle (1024-byte atoms of 8 rows x 128 bytes,
// 16-byte chunk c of row r stored at chunk c ^ (r % 8)), so that the eight
// threads of a quarter-warp storing one 128-byte row hit distinct banks.
//  G  (A, K-major):  rows m = 2k+b (128), K = 2n+a (128) = 2 atoms of 64
//  B1 (B, MN-major): rows = K (128), N = n2 (64 = one 128-byte row)
//  B2 (B, K-major):  rows n = k1 (64), K = 2*n2+a (128) = 2 atoms of 64
constexpr uint32_t G_KATOM = 16384;   // 16 row groups x 1024
constexpr uint32_t B2_KATOM = 8192;   //  8 row groups x 1024
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
__host__ __device__ constexpr uint32_t g_off(int m, int kk) { return kmaj_off(m, kk, G_KATOM); }

// Tables: G planes (hi, lo with the 16x scale; bf16 unscaled) in the exact
// shared-memory image, and T[m] = W4096^m; all from FP64 sincospi.
__global__ void k_tc_tables(__half* g_hi, __half* g_lo, __nv_bfloat16* g_bf, float2* tw) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // 0 .. 128*128-1
    if (idx < 128 * 128) {
        const int m = idx / 128, kk = idx % 128;
        const int k = m >> 1, b = m & 1, n = kk >> 1, a = kk & 1;
        double s, c;
        sincospi(-2.0 * (double)((n * k) % TC_R) / (double)TC_R, &s, &c);  // W64^(nk) = c + i s
        // out re = c*xr - s*xi ; out im = s*xr + c*xi
        const double gv = (b == 0) ? (a == 0 ? c : -s) : (a == 0 ? s : c);
        const uint32_t o = g_off(m, kk) / 2;
        const float gs = (float)(gv * TC_GSCALE);
        const __half h = __float2half_rn(gs);
        g_hi[o] = h;
        g_lo[o] = __float2half_rn(gs - __half2float(h));
        g_bf[o] = __float2bfloat16_rn((float)gv);
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

// ---- four pipelines per CTA -------------------------------------------------
//
// One CTA of 512 threads per SM holds the DFT-64 operand once and runs four
// independent 128-thread pipelines, each with its own line, B operand buffers
// (32 KB), TMEM columns (D1, D2), commit mbarrier and named barrier: four
// lines in flight per SM where two CTAs of one pipeline each hold two (and
// two copies of the operand).  A pipeline's four warps cover the 128 TMEM
// lanes, each walking both 32-column halves of D1 and D2; lines are loaded
// directly into registers, the pipeline's next line prefetched into L2 one
// line ahead (split 33.1 -> 34.6 M, BF16 45.9 -> 48.9 M transforms/s).
constexpr int TQ_PIPES = 4, TQ_PT = 128, TQ_THREADS = TQ_PIPES * TQ_PT;
constexpr uint32_t TQ_B = 65536, TQ_BSTRIDE = 32768;          // pipeline p: B hi at TQ_B + p*TQ_BSTRIDE, lo +16 KB
constexpr uint32_t TQ_T1 = TQ_B + TQ_PIPES * TQ_BSTRIDE;      // W4096^(i*k1), i < 16: 8 KB
constexpr uint32_t TQ_T0 = TQ_T1 + 8192;                      // W4096^(16*j*k1), j < 4: 2 KB
constexpr uint32_t TQ_SMEM = TQ_T0 + 2048 + 1024;             // + alignment slack

template <bool SPLIT>
__device__ __forceinline__ void store_chunk_b(uint8_t* bhi, uint32_t off, const float (&x)[8]) {
    if constexpr (SPLIT) {
        __align__(16) __half hi[8];
        __align__(16) __half lo[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            hi[i] = __float2half_rn(x[i]);
            lo[i] = __float2half_rn(x[i] - __half2float(hi[i]));
        }
        *reinterpret_cast<uint4*>(bhi + off) = *reinterpret_cast<const uint4*>(hi);
        *reinterpret_cast<uint4*>(bhi + 16384 + off) = *reinterpret_cast<const uint4*>(lo);
    } else {
        __align__(16) __nv_bfloat16 bf[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) bf[i] = __float2bfloat16_rn(x[i]);
        *reinterpret_cast<uint4*>(bhi + off) = *reinterpret_cast<const uint4*>(bf);
    }
}

// D (+)= G * B over K = 128 with this pipeline's B planes at b_addr (lo +16 KB)
template <bool SPLIT, bool B_MN>
__device__ __forceinline__ void issue_product_q(uint32_t d_tmem, uint32_t g_addr, uint32_t b_addr, uint32_t idesc) {
    constexpr int NPROD = SPLIT ? 3 : 1;
#pragma unroll
    for (int pr = 0; pr < NPROD; ++pr) {
        const uint32_t ga = g_addr + (pr == 2 ? SM_G1 : SM_G0);
        const uint32_t bb = b_addr + (pr == 1 ? 16384u : 0u);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint64_t ad = tc::smem_desc(ga + (j / 4) * G_KATOM + (j % 4) * 32, 16, ATOM_SBO, tc::LAYOUT_SW128);
            const uint64_t bd =
                B_MN ? tc::smem_desc(bb + 2 * j * ATOM_SBO, 16384, ATOM_SBO, tc::LAYOUT_SW128)
                     : tc::smem_desc(bb + (j / 4) * B2_KATOM + (j % 4) * 32, 16, ATOM_SBO, tc::LAYOUT_SW128);
            tc::mma_f16_ss(d_tmem, ad, bd, idesc, (pr > 0 || j > 0) ? 1u : 0u);
        }
    }
}

// bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned) into L2
__device__ __forceinline__ void prefetch_l2(const void* g, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(g), "r"(bytes) : "memory");
}

__device__ __forceinline__ void pipe_sync(int p) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + p), "r"(TQ_PT) : "memory");
}

template <bool SPLIT, bool INV>
__global__ void __launch_bounds__(TQ_THREADS, 1)
    k_fft4096_tcq(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
                  const uint4* __restrict__ gimg, const float2* __restrict__ tw, int* dev_err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t mbar[TQ_PIPES];
    __shared__ uint32_t tmem_base_sh;
    __shared__ float red1[TQ_PIPES][4];
    __shared__ int abort_sh[TQ_PIPES];

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int p = warp >> 2;              // pipeline
    const int q = warp & 3;               // this warp's TMEM lane quarter
    const int ptid = tid & (TQ_PT - 1);   // thread within the pipeline
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_u32(smem);
    constexpr uint32_t FMT = SPLIT ? 0u : 1u;
    constexpr uint32_t IDESC1 = tc::idesc_f16(FMT, 1u, 128, 64);
    constexpr uint32_t IDESC2 = tc::idesc_f16(FMT, 0u, 128, 64);

    constexpr int GWORDS = (SPLIT ? 65536 : 32768) / 16;
    for (int i = tid; i < GWORDS; i += TQ_THREADS) reinterpret_cast<uint4*>(smem)[i] = __ldg(gimg + i);
    float2* t1 = reinterpret_cast<float2*>(smem + TQ_T1);
    float2* t0 = reinterpret_cast<float2*>(smem + TQ_T0);
    for (int i = tid; i < 16 * 64; i += TQ_THREADS) t1[i] = __ldg(tw + ((i >> 6) * (i & 63)));
    for (int i = tid; i < 4 * 64; i += TQ_THREADS) t0[i] = __ldg(tw + (16 * (i >> 6) * (i & 63)));
    if (tid < TQ_PIPES) {
        mbar_init(&mbar[tid], 1);
        abort_sh[tid] = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base_sh, 512);
        tc::tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t d1 = tmem_base_sh + (uint32_t)p * 128u, d2 = d1 + 64u;
    uint8_t* bp = smem + TQ_B + (uint32_t)p * TQ_BSTRIDE;
    const uint32_t baddr = sbase + TQ_B + (uint32_t)p * TQ_BSTRIDE;

    const int m = 32 * q + lane;  // TMEM lane = D row = 2k + b
    const int kk_ = m >> 1, bsel = m & 1;
    const uint32_t lane_off = (uint32_t)(32 * q) << 16;

    uint32_t phase = 0;
    bool aborted = false;
    const long long fstep = (long long)gridDim.x * TQ_PIPES;
    for (long long f = (long long)blockIdx.x * TQ_PIPES + p; f < batch; f += fstep) {
        // this pipeline's next line to L2 while this one goes through both stages
        if (ptid == 0 && f + fstep < batch) prefetch_l2(in + (size_t)(f + fstep) * TC_N, TC_N * sizeof(float2));
        // ---- the line, its scale, the stage-1 operand (MN-major) ----
        float4 cur[16];
        const float4* src = reinterpret_cast<const float4*>(in + (size_t)f * TC_N);
#pragma unroll
        for (int it = 0; it < 4; ++it)
#pragma unroll
            for (int j = 0; j < 4; ++j) cur[4 * it + j] = __ldcs(src + 4 * (ptid + TQ_PT * it) + j);
        if constexpr (INV) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                cur[i].y = -cur[i].y;
                cur[i].w = -cur[i].w;
            }
        }
        float s1 = 1.f;
        if constexpr (SPLIT) {
            float mx = 0.f;
#pragma unroll
            for (int i = 0; i < 16; ++i)
                mx = fmaxf(mx, fmaxf(fmaxf(fabsf(cur[i].x), fabsf(cur[i].y)), fmaxf(fabsf(cur[i].z), fabsf(cur[i].w))));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0) red1[p][q] = mx;
            pipe_sync(p);
            s1 = line_scale(fmaxf(fmaxf(red1[p][0], red1[p][1]), fmaxf(red1[p][2], red1[p][3])));
        }
#pragma unroll
        for (int it = 0; it < 4; ++it) {
            const int item = ptid + TQ_PT * it;  // (n1, c): n2 = 8c .. 8c+7
            const int n1 = item >> 3, c = item & 7;
            float re[8], im[8];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float4 v = cur[4 * it + j];
                re[2 * j] = v.x * s1;
                im[2 * j] = v.y * s1;
                re[2 * j + 1] = v.z * s1;
                im[2 * j + 1] = v.w * s1;
            }
            store_chunk_b<SPLIT>(bp, mnmaj_off(8 * c, 2 * n1), re);
            store_chunk_b<SPLIT>(bp, mnmaj_off(8 * c, 2 * n1 + 1), im);
        }
        fence_proxy_async_smem();
        tc::fence_before_sync();
        pipe_sync(p);

        // ---- stage 1 ----
        if (ptid == 0) {
            tc::fence_after_sync();
            issue_product_q<SPLIT, true>(d1, sbase, baddr, IDESC1);
            tc::mma_commit(&mbar[p]);
            if (!mbar_wait(&mbar[p], phase)) abort_sh[p] = 1;
        }
        phase ^= 1u;
        pipe_sync(p);
        if (abort_sh[p]) {
            aborted = true;
            break;
        }
        tc::fence_after_sync();

        // ---- epilogue 1: unscale, pair re/im, twiddle, scale, stage-2 operand (K-major) ----
        const float inv1 = 1.f / ((SPLIT ? TC_GSCALE : 1.f) * s1);
        const float s2 = SPLIT ? s1 * (1.f / 64.f) : 1.f;
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            float2 z[16];
            {
                float v[32];
                tc::tmem_ld32(d1 + lane_off + 32 * h, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const float send = bsel ? v[i] : v[16 + i];
                    const float r = __shfl_xor_sync(0xffffffffu, send, 1);
                    z[i] = bsel ? make_float2(r * inv1, v[16 + i] * inv1) : make_float2(v[i] * inv1, r * inv1);
                }
            }
            const int n2_0 = 32 * h + 16 * bsel;
            const float2 w0 = t0[(n2_0 >> 4) * 64 + kk_];
#pragma unroll
            for (int i = 0; i < 16; ++i) z[i] = cmul(z[i], cmul(w0, t1[i * 64 + kk_]));
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                float x[8];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    x[2 * j] = z[4 * qq + j].x * s2;
                    x[2 * j + 1] = z[4 * qq + j].y * s2;
                }
                store_chunk_b<SPLIT>(bp, kmaj_off(kk_, 2 * (n2_0 + 4 * qq), B2_KATOM), x);
            }
        }
        fence_proxy_async_smem();
        tc::fence_before_sync();
        pipe_sync(p);

        // ---- stage 2 ----
        if (ptid == 0) {
            tc::fence_after_sync();
            issue_product_q<SPLIT, false>(d2, sbase, baddr, IDESC2);
            tc::mma_commit(&mbar[p]);
            if (!mbar_wait(&mbar[p], phase)) abort_sh[p] = 1;
        }
        phase ^= 1u;
        pipe_sync(p);
        if (abort_sh[p]) {
            aborted = true;
            break;
        }
        tc::fence_after_sync();

        // ---- epilogue 2: unscale, pair re/im, store X[k1 + 64 k2] ----
        const float inv2 = (INV ? 1.f / (float)TC_N : 1.f) / ((SPLIT ? TC_GSCALE : 1.f) * s2);
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            float v[32];
            tc::tmem_ld32(d2 + lane_off + 32 * h, v);
            float4 o[8];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float send = bsel ? v[i] : v[16 + i];
                const float r = __shfl_xor_sync(0xffffffffu, send, 1);
                float2 y = bsel ? make_float2(r * inv2, v[16 + i] * inv2) : make_float2(v[i] * inv2, r * inv2);
                if constexpr (INV) y.y = -y.y;
                if (i & 1) {
                    o[i >> 1].z = y.x;
                    o[i >> 1].w = y.y;
                } else {
                    o[i >> 1].x = y.x;
                    o[i >> 1].y = y.y;
                }
            }
            const int k1_0 = 32 * h + 16 * bsel;  // k2 = kk_
            float4* dst = reinterpret_cast<float4*>(out + (size_t)f * TC_N + TC_R * kk_ + k1_0);
#pragma unroll
            for (int i = 0; i < 8; ++i) __stcs(dst + i, o[i]);
        }
        tc::fence_before_sync();
        pipe_sync(p);  // this pipeline's TMEM columns and B buffers are free for its next line
    }

    if (aborted && ptid == 0) {
        report_device_error(dev_err, DEV_ERR_MMA_TIMEOUT);
        mbar_wait(&mbar[p], phase ^ 1u);  // bounded: let an MMA still in flight finish
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_base_sh, 512);
    }
}

template <bool SPLIT, bool INV>
cudaError_t launch_tcq(const float2* in, float2* out, long long batch, const uint4* gimg, const float2* tw,
                       int* dev_err, int sms, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(k_fft4096_tcq<SPLIT, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TQ_SMEM);
    if (e != cudaSuccess) return e;
    long long blocks = (batch + TQ_PIPES - 1) / TQ_PIPES;
    if (blocks > sms) blocks = sms;
    if (blocks <= 0) return cudaSuccess;
    k_fft4096_tcq<SPLIT, INV><<<(unsigned)blocks, TQ_THREADS, TQ_SMEM, s>>>(in, out, batch, gimg, tw, dev_err);
    return cudaGetLastError();
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
        e = inv ? launch_tcq<true, true>(in, out, batch, g_split, p->tc.tw, err, sms, s)
                : launch_tcq<true, false>(in, out, batch, g_split, p->tc.tw, err, sms, s);
    else
        e = inv ? launch_tcq<false, true>(in, out, batch, g_bf, p->tc.tw, err, sms, s)
                : launch_tcq<false, false>(in, out, batch, g_bf, p->tc.tw, err, sms, s);
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
