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
// One CTA of 256 threads (8 warps) transforms one line at a time, 2 CTAs per
// SM; the next line's loads are issued before the current line's tensor-core
// work so they overlap it, and its maximum is published at the barrier that
// ends the current line.  The stage-2 scale is s1/64 (a DFT-64 grows
// magnitudes by at most 64), so no reduction sits between the two products.  The single thread that issues the MMAs waits on
// the commit mbarrier with a time limit; a timeout sets the device error word
// and the CTA leaves its loop, frees its TMEM and returns.
#include "capi_internal.h"
#include "fft_common.cuh"
#include "tcgen05.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace mfft {

namespace {

constexpr int TC_N = 4096;
constexpr int TC_R = 64;
constexpr int TC_THREADS = 256;
constexpr float TC_GSCALE = 16.0f;  // FP16 split: G stored as 16 * DFT-64
constexpr int TC_LINE_EXP = 14;     // FP16 split: line scaled so |max| < 2^14

// shared-memory byte offsets from a 1024-byte aligned base (dynamic)
constexpr uint32_t SM_G0 = 0;          // G hi (or bf16) : 128 x 128 halves = 32 KB
constexpr uint32_t SM_G1 = 32768;      // G lo
constexpr uint32_t SM_B0 = 65536;      // B hi (or bf16) : 128 x 64 halves = 16 KB
constexpr uint32_t SM_B1 = 81920;      // B lo
constexpr uint32_t SM_T1 = 98304;      // W4096^(i*k1), i < 16, k1 < 64: 8 KB
constexpr uint32_t SM_T0 = 106496;     // W4096^(16*j*k1), j < 4, k1 < 64: 2 KB
constexpr uint32_t SM_BYTES = 108544 + 1024;  // + alignment slack
constexpr uint32_t TMEM_COLS = 128;    // D1: columns [0, 64), D2: [64, 128)

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

// 8 values -> one 16-byte chunk of hi (and lo) halves / bf16
template <bool SPLIT>
__device__ __forceinline__ void store_chunk(uint8_t* smem, uint32_t off, const float (&x)[8]) {
    if constexpr (SPLIT) {
        __align__(16) __half hi[8];
        __align__(16) __half lo[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            hi[i] = __float2half_rn(x[i]);
            lo[i] = __float2half_rn(x[i] - __half2float(hi[i]));
        }
        *reinterpret_cast<uint4*>(smem + SM_B0 + off) = *reinterpret_cast<const uint4*>(hi);
        *reinterpret_cast<uint4*>(smem + SM_B1 + off) = *reinterpret_cast<const uint4*>(lo);
    } else {
        __align__(16) __nv_bfloat16 bf[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) bf[i] = __float2bfloat16_rn(x[i]);
        *reinterpret_cast<uint4*>(smem + SM_B0 + off) = *reinterpret_cast<const uint4*>(bf);
    }
}

// D (+)= G * B over K = 128 (8 steps of 16): three products for the split.
// K step j: K-major operands advance (j/4) atoms plus (j%4)*32 bytes inside
// the 128-byte row; the MN-major B1 advances two 8-row groups.
template <bool SPLIT, bool B_MN>
__device__ __forceinline__ void issue_product(uint32_t d_tmem, uint32_t smem_base, uint32_t idesc) {
    constexpr int NPROD = SPLIT ? 3 : 1;
#pragma unroll
    for (int p = 0; p < NPROD; ++p) {
        const uint32_t ga = smem_base + (p == 2 ? SM_G1 : SM_G0);
        const uint32_t bb = smem_base + (p == 1 ? SM_B1 : SM_B0);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint64_t ad = tc::smem_desc(ga + (j / 4) * G_KATOM + (j % 4) * 32, 16, ATOM_SBO, tc::LAYOUT_SW128);
            const uint64_t bd =
                B_MN ? tc::smem_desc(bb + 2 * j * ATOM_SBO, 16384, ATOM_SBO, tc::LAYOUT_SW128)
                     : tc::smem_desc(bb + (j / 4) * B2_KATOM + (j % 4) * 32, 16, ATOM_SBO, tc::LAYOUT_SW128);
            tc::mma_f16_ss(d_tmem, ad, bd, idesc, (p > 0 || j > 0) ? 1u : 0u);
        }
    }
}

template <bool SPLIT, bool INV>
__global__ void __launch_bounds__(TC_THREADS, 2)
    k_fft4096_tc(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
                 const uint4* __restrict__ gimg, const float2* __restrict__ tw, int* dev_err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ float red1[TC_THREADS / 32];
    __shared__ int abort_sh;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    // swizzle atoms need 1024-byte alignment
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_u32(smem);
    constexpr uint32_t FMT = SPLIT ? 0u : 1u;
    constexpr uint32_t IDESC1 = tc::idesc_f16(FMT, 1u, 128, 64);  // B MN-major
    constexpr uint32_t IDESC2 = tc::idesc_f16(FMT, 0u, 128, 64);  // B K-major

    // G planes into shared memory (32 KB per plane)
    constexpr int GWORDS = (SPLIT ? 65536 : 32768) / 16;
    for (int i = tid; i < GWORDS; i += TC_THREADS)
        reinterpret_cast<uint4*>(smem)[i] = __ldg(gimg + i);
    // stage twiddles W4096^(n2*k1), n2 = 16*j + i: T0[j][k1] * T1[i][k1], so a
    // warp (consecutive k1) reads consecutive shared-memory words
    float2* t1 = reinterpret_cast<float2*>(smem + SM_T1);
    float2* t0 = reinterpret_cast<float2*>(smem + SM_T0);
    for (int i = tid; i < 16 * 64; i += TC_THREADS) t1[i] = __ldg(tw + ((i >> 6) * (i & 63)));
    for (int i = tid; i < 4 * 64; i += TC_THREADS) t0[i] = __ldg(tw + (16 * (i >> 6) * (i & 63)));
    if (tid == 0) {
        mbar_init(&mbar, 1);
        abort_sh = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base_sh, TMEM_COLS);
        tc::tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base_sh;
    const uint32_t d1 = tmem, d2 = tmem + 64;

    // epilogue geometry: warp -> lane quarter q, column half h
    const int q = warp & 3, h = warp >> 2;
    const int m = 32 * q + lane;        // TMEM lane = D row = 2k + b
    const int kk_ = m >> 1, bsel = m & 1;
    const uint32_t lane_off = (uint32_t)(32 * q) << 16;

    float4 cur[8];
    auto load_line = [&](long long f) {
        const float4* src = reinterpret_cast<const float4*>(in + (size_t)f * TC_N);
#pragma unroll
        for (int it = 0; it < 2; ++it)
#pragma unroll
            for (int j = 0; j < 4; ++j) cur[4 * it + j] = __ldcs(src + 4 * (tid + TC_THREADS * it) + j);
    };

    // per-warp partial max of the line in `cur`, published through red1 by
    // the barrier that precedes its use
    auto publish_max = [&]() {
        float mx = 0.f;
#pragma unroll
        for (int i = 0; i < 8; ++i)
            mx = fmaxf(mx, fmaxf(fmaxf(fabsf(cur[i].x), fabsf(cur[i].y)), fmaxf(fabsf(cur[i].z), fabsf(cur[i].w))));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) red1[warp] = mx;
    };

    uint32_t phase = 0;
    long long f = blockIdx.x;
    if (f < batch) {
        load_line(f);
        if constexpr (SPLIT) publish_max();
    }
    __syncthreads();
    for (; f < batch; f += gridDim.x) {
        // ---- stage-1 operand: scale, split, write B (MN-major) ----
        if constexpr (INV) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                cur[i].y = -cur[i].y;
                cur[i].w = -cur[i].w;
            }
        }
        float s1 = 1.f;
        if constexpr (SPLIT) {
            float m = red1[0];
#pragma unroll
            for (int w = 1; w < TC_THREADS / 32; ++w) m = fmaxf(m, red1[w]);
            s1 = line_scale(m);
        }
#pragma unroll
        for (int it = 0; it < 2; ++it) {
            const int item = tid + TC_THREADS * it;  // (n1, c): n2 = 8c .. 8c+7
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
            // MN-major rows kk = 2*n1 (re) and 2*n1 + 1 (im), chunk c of n2
            store_chunk<SPLIT>(smem, mnmaj_off(8 * c, 2 * n1), re);
            store_chunk<SPLIT>(smem, mnmaj_off(8 * c, 2 * n1 + 1), im);
        }
        // prefetch the next line: in flight during the tensor-core work
        if (f + gridDim.x < batch) load_line(f + gridDim.x);
        fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();

        // ---- stage 1 on the tensor cores ----
        if (tid == 0) {
            tc::fence_after_sync();
            issue_product<SPLIT, true>(d1, sbase, IDESC1);
            tc::mma_commit(&mbar);
            if (!mbar_wait(&mbar, phase)) abort_sh = 1;
        }
        phase ^= 1u;
        __syncthreads();
        if (abort_sh) break;
        tc::fence_after_sync();

        // ---- epilogue 1: unscale, pair re/im, twiddle, scale, write B (K-major) ----
        float2 z[16];
        {
            float v[32];
            tc::tmem_ld32(d1 + lane_off + 32 * h, v);
            const float inv1 = 1.f / ((SPLIT ? TC_GSCALE : 1.f) * s1);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float send = bsel ? v[i] : v[16 + i];
                const float r = __shfl_xor_sync(0xffffffffu, send, 1);
                z[i] = bsel ? make_float2(r * inv1, v[16 + i] * inv1) : make_float2(v[i] * inv1, r * inv1);
            }
        }
        const int n2_0 = 32 * h + 16 * bsel;  // this thread's n2 range; k1 = kk_
        {
            const float2 w0 = t0[(n2_0 >> 4) * 64 + kk_];
#pragma unroll
            for (int i = 0; i < 16; ++i) z[i] = cmul(z[i], cmul(w0, t1[i * 64 + kk_]));
        }
        // a DFT-64 grows magnitudes by at most 64: s1 / 64 keeps |Z| s2 < 2^14
        // without a second reduction over the line
        const float s2 = SPLIT ? s1 * (1.f / 64.f) : 1.f;
        {
            // K-major row nn = k1, K = 2*n2 + a: 4 chunks of 8 (4 complex values)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                float x[8];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    x[2 * j] = z[4 * qq + j].x * s2;
                    x[2 * j + 1] = z[4 * qq + j].y * s2;
                }
                store_chunk<SPLIT>(smem, kmaj_off(kk_, 2 * (n2_0 + 4 * qq), B2_KATOM), x);
            }
        }
        fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();

        // ---- stage 2 on the tensor cores ----
        if (tid == 0) {
            tc::fence_after_sync();
            issue_product<SPLIT, false>(d2, sbase, IDESC2);
            tc::mma_commit(&mbar);
            if (!mbar_wait(&mbar, phase)) abort_sh = 1;
        }
        phase ^= 1u;
        __syncthreads();
        if (abort_sh) break;
        tc::fence_after_sync();

        // ---- epilogue 2: unscale, pair re/im, store X[k1 + 64 k2] ----
        {
            float v[32];
            tc::tmem_ld32(d2 + lane_off + 32 * h, v);
            const float inv2 = (INV ? 1.f / (float)TC_N : 1.f) / ((SPLIT ? TC_GSCALE : 1.f) * s2);
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
        if constexpr (SPLIT) {
            if (f + gridDim.x < batch) publish_max();  // the prefetched line
        }
        tc::fence_before_sync();
        __syncthreads();  // TMEM and B are free for the next line; red1 published
    }

    if (abort_sh && tid == 0) {
        report_device_error(dev_err, DEV_ERR_MMA_TIMEOUT);
        mbar_wait(&mbar, phase ^ 1u);  // bounded: let an MMA still in flight finish
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, TMEM_COLS);
    }
}

template <bool SPLIT, bool INV>
cudaError_t launch_tc(const float2* in, float2* out, long long batch, const uint4* gimg, const float2* tw,
                      int* dev_err, int sms, cudaStream_t s) {
    // the shared-memory opt-in is a per-device attribute: set it on the
    // current device at every call (a few microseconds)
    cudaError_t e = cudaFuncSetAttribute(k_fft4096_tc<SPLIT, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_BYTES);
    if (e != cudaSuccess) return e;
    long long blocks = (long long)sms * 2;
    if (blocks > batch) blocks = batch;
    if (blocks <= 0) return cudaSuccess;
    k_fft4096_tc<SPLIT, INV><<<(unsigned)blocks, TC_THREADS, SM_BYTES, s>>>(in, out, batch, gimg, tw, dev_err);
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
        e = inv ? launch_tc<true, true>(in, out, batch, g_split, p->tc.tw, err, sms, s)
                : launch_tc<true, false>(in, out, batch, g_split, p->tc.tw, err, sms, s);
    else
        e = inv ? launch_tc<false, true>(in, out, batch, g_bf, p->tc.tw, err, sms, s)
                : launch_tc<false, false>(in, out, batch, g_bf, p->tc.tw, err, sms, s);
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
