// conv_fp16.cu -- the FusedConvolver's FP16 precision modes (fft = 4096).
//
// Reference: FusedConvolver.Precision (Sources/MetalFFT/DSP/
// FusedConvolver.swift:27-36) selects one of three FP16 variants of the fused
// FFT -> * H -> IFFT kernel (Resources/fft_fused_convolve_fp16.metal:160-498):
//   float16Storage  intermediate values stored as half2 between passes,
//                   butterflies and twiddles in FP32 (:316-350);
//   float16Mixed    the same storage, every twiddle multiply and the filter
//                   multiply in FP16, additions in FP32 (:356-498);
//   float16Pure     all butterfly arithmetic in FP16 (:160-190).
// In each the spectrum X and the product X*H are stored as half2 and the
// inverse output leaves in FP32.
//
// Here the same three policies run inside the overlap-add walker of the FP32
// forward kernel (conv.cu: two blocks per complex line, overlap carried in
// shared memory): 16 elements per thread, three radix-16 passes, the two
// exchanges through half2 shared memory (17 KB per line instead of 34 KB).
// Range: H is multiplied by 2^-6 on load and the inverse's 1/N becomes 2^6/N
// (both exact power-of-two scalings), so X*H and the inverse's partial sums
// stay 64x below the FP16 limit that the reference's order of scaling (1/N
// at the very end, :141-147) runs into for |x*h| of a few units.
#include <cuda_fp16.h>

#include "capi_internal.h"
#include "stockham.cuh"

namespace mfft {

namespace {

constexpr int FH_N = 4096, FH_E = 16, FH_T = FH_N / FH_E;
constexpr float FH_HSCALE = 0.015625f;  // 2^-6 on H
using FhPlan = SPlan<FH_N, FH_E>;

__device__ __forceinline__ __half2 h2(float2 a) { return __float22half2_rn(a); }
__device__ __forceinline__ float2 f2(__half2 a) { return __half22float2(a); }
__device__ __forceinline__ float2 round_h(float2 a) { return f2(h2(a)); }
__device__ __forceinline__ int hpad(int i) { return i + (i >> 5); }
// complex product in FP16
__device__ __forceinline__ __half2 hcmul(__half2 a, __half2 b) { return __hcmadd(a, b, __float2half2_rn(0.f)); }

constexpr float FH_R2 = 0.70710678118654752440f;  // cos(pi/4)
constexpr float FH_C8 = 0.92387953251128675613f;  // cos(pi/8)
constexpr float FH_S8 = 0.38268343236508977173f;  // sin(pi/8)

// float16Storage: FP32 arithmetic; values cross the exchange as half2.
struct ArStorage {
    using V = float2;
    using W = float2;
    static __device__ __forceinline__ V add(V a, V b) { return cadd(a, b); }
    static __device__ __forceinline__ V sub(V a, V b) { return csub(a, b); }
    static __device__ __forceinline__ V mi(V a) { return mul_mi(a); }
    static __device__ __forceinline__ V rot(V a, float c, float s) { return mul_c(a, c, s); }
    static __device__ __forceinline__ W tw(float2 w) { return w; }
    static __device__ __forceinline__ W wmul(W a, W b) { return cmul(a, b); }
    static __device__ __forceinline__ V tmul(V a, W w) { return cmul(a, w); }
    static __device__ __forceinline__ void store(__half2* p, V v) { *p = h2(v); }
    static __device__ __forceinline__ V load(const __half2* p) { return f2(*p); }
};
// float16Mixed: FP32 additions; every rotation and twiddle multiply in FP16.
struct ArMixed : ArStorage {
    using W = __half2;
    static __device__ __forceinline__ W tw(float2 w) { return h2(w); }
    static __device__ __forceinline__ W wmul(W a, W b) { return hcmul(a, b); }
    static __device__ __forceinline__ V tmul(V a, W w) { return f2(hcmul(h2(a), w)); }
    static __device__ __forceinline__ V rot(V a, float c, float s) { return tmul(a, h2(make_float2(c, s))); }
};
// float16Pure: all arithmetic in FP16.
struct ArPure {
    using V = __half2;
    using W = __half2;
    static __device__ __forceinline__ V add(V a, V b) { return __hadd2(a, b); }
    static __device__ __forceinline__ V sub(V a, V b) { return __hsub2(a, b); }
    // -i (x + i y) = y - i x
    static __device__ __forceinline__ V mi(V a) { return __hmul2(__lowhigh2highlow(a), __floats2half2_rn(1.f, -1.f)); }
    static __device__ __forceinline__ V rot(V a, float c, float s) { return hcmul(a, __floats2half2_rn(c, s)); }
    static __device__ __forceinline__ W tw(float2 w) { return h2(w); }
    static __device__ __forceinline__ W wmul(W a, W b) { return hcmul(a, b); }
    static __device__ __forceinline__ V tmul(V a, W w) { return hcmul(a, w); }
    static __device__ __forceinline__ void store(__half2* p, V v) { *p = v; }
    static __device__ __forceinline__ V load(const __half2* p) { return *p; }
};

// 4-point DFT on v[0], v[S], v[2S], v[3S] (forward sign), natural order
template <class A, int S>
__device__ __forceinline__ void hdft4(typename A::V* v) {
    using V = typename A::V;
    const V t0 = A::add(v[0], v[2 * S]), t1 = A::sub(v[0], v[2 * S]);
    const V t2 = A::add(v[S], v[3 * S]), t3 = A::mi(A::sub(v[S], v[3 * S]));
    v[0] = A::add(t0, t2);
    v[2 * S] = A::sub(t0, t2);
    v[S] = A::add(t1, t3);
    v[3 * S] = A::sub(t1, t3);
}

// 16-point DFT as 4 x 4 (n = 4 n1 + n2, k = k1 + 4 k2) with the W16
// rotations of the policy
template <class A>
__device__ __forceinline__ void hdft16(typename A::V (&v)[FH_E]) {
    using V = typename A::V;
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) hdft4<A, 4>(v + n2);
    v[5] = A::rot(v[5], FH_C8, -FH_S8);    // W^1
    v[9] = A::rot(v[9], FH_R2, -FH_R2);    // W^2
    v[13] = A::rot(v[13], FH_S8, -FH_C8);  // W^3
    v[6] = A::rot(v[6], FH_R2, -FH_R2);    // W^2
    v[10] = A::mi(v[10]);                  // W^4
    v[14] = A::rot(v[14], -FH_R2, -FH_R2); // W^6
    v[7] = A::rot(v[7], FH_S8, -FH_C8);    // W^3
    v[11] = A::rot(v[11], -FH_R2, -FH_R2); // W^6
    v[15] = A::rot(v[15], -FH_C8, FH_S8);  // W^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) hdft4<A, 1>(v + 4 * k1);
    V a[FH_E];
#pragma unroll
    for (int i = 0; i < FH_E; ++i) a[i] = v[i];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = a[4 * k1 + k2];
}

// v[r] *= w^r from the twiddle row {w, w^2, w^4, w^8}; the other powers are
// products in the policy's twiddle arithmetic (the reference forms w^2, w^3
// the same way: fft_fused_convolve_fp16.metal:55-60, 362-367)
template <class A>
__device__ __forceinline__ void htwiddle(typename A::V (&v)[FH_E], const float2* __restrict__ row) {
    using W = typename A::W;
    const float4 q0 = __ldg(reinterpret_cast<const float4*>(row));
    const float4 q1 = __ldg(reinterpret_cast<const float4*>(row) + 1);
    const W w1 = A::tw(make_float2(q0.x, q0.y)), w2 = A::tw(make_float2(q0.z, q0.w));
    const W w4 = A::tw(make_float2(q1.x, q1.y)), w8 = A::tw(make_float2(q1.z, q1.w));
    const W w3 = A::wmul(w1, w2), w5 = A::wmul(w1, w4), w6 = A::wmul(w2, w4), w7 = A::wmul(w3, w4);
    v[1] = A::tmul(v[1], w1);
    v[2] = A::tmul(v[2], w2);
    v[3] = A::tmul(v[3], w3);
    v[4] = A::tmul(v[4], w4);
    v[5] = A::tmul(v[5], w5);
    v[6] = A::tmul(v[6], w6);
    v[7] = A::tmul(v[7], w7);
    v[8] = A::tmul(v[8], w8);
    v[9] = A::tmul(v[9], A::wmul(w1, w8));
    v[10] = A::tmul(v[10], A::wmul(w2, w8));
    v[11] = A::tmul(v[11], A::wmul(w3, w8));
    v[12] = A::tmul(v[12], A::wmul(w4, w8));
    v[13] = A::tmul(v[13], A::wmul(w5, w8));
    v[14] = A::tmul(v[14], A::wmul(w6, w8));
    v[15] = A::tmul(v[15], A::wmul(w7, w8));
}

// pass P of the 3-pass radix-16 Stockham FFT of 4096 points, 256 threads:
// on entry v[m] = element t + 256 m of the pass input; exchanges through the
// half2 line `buf` (padded index hpad: one spare 4-byte slot per 32, so a
// warp reading 32 consecutive elements hits 32 distinct banks)
template <class A, int P>
__device__ __forceinline__ void hpass(typename A::V (&v)[FH_E], int t, __half2* buf, const float2* __restrict__ tw) {
    constexpr int NS = FhPlan::span(P);
    if constexpr (NS > 1) htwiddle<A>(v, tw + FhPlan::twoff(P) + (t & (NS - 1)) * FhPlan::twrow(FH_E));
    hdft16<A>(v);
    if constexpr (P + 1 < FhPlan::NPASS) {
        const int k = t & (NS - 1);
        const int d = (t - k) * FH_E + k;
#pragma unroll
        for (int r = 0; r < FH_E; ++r) A::store(buf + hpad(d + r * NS), v[r]);
        __syncthreads();
#pragma unroll
        for (int m = 0; m < FH_E; ++m) v[m] = A::load(buf + hpad(t + m * FH_T));
        __syncthreads();
        hpass<A, P + 1>(v, t, buf, tw);
    }
}

// number of valid samples in a window of `cap` when `avail` remain (0 .. cap)
__device__ __forceinline__ int fh_count(long long avail, int cap) {
    return avail <= 0 ? 0 : (avail >= cap ? cap : (int)avail);
}

template <int MODE>
struct FhPolicy;
template <>
struct FhPolicy<MFFT_CONV_FP16_STORAGE> {
    using A = ArStorage;
};
template <>
struct FhPolicy<MFFT_CONV_FP16_MIXED> {
    using A = ArMixed;
};
template <>
struct FhPolicy<MFFT_CONV_FP16_PURE> {
    using A = ArPure;
};

constexpr int FH_XCH = FH_N + FH_N / 32;                      // half2 slots of the exchange line
constexpr int FH_SMEM = FH_XCH * 4 + 2 * FH_N * 4;               // half2 exchange + two FP32 overlap rows

// Same walker contract as the FP32 forward kernel: unit = CTA owns block
// pairs [p0, p1) of the nout output blocks, recomputes `warm_blocks` earlier
// blocks for its first overlap, writes y[b*hop, (b+1)*hop) once per block.
template <int MODE>
__global__ void __launch_bounds__(FH_T, 2)
    k_conv_fwd_h(const float* __restrict__ x, long long nx, float* __restrict__ y, long long ny,
                 const float2* __restrict__ H, const float2* __restrict__ tw, int hop, long long npairs,
                 long long pairs_per_unit, int warm_blocks) {
    using A = typename FhPolicy<MODE>::A;
    using V = typename A::V;
    extern __shared__ __align__(16) unsigned char fh_smem[];
    __half2* buf = reinterpret_cast<__half2*>(fh_smem);
    float* acc0 = reinterpret_cast<float*>(fh_smem + FH_XCH * 4);
    float* acc1 = acc0 + FH_N;
    const int t = threadIdx.x;
    const long long unit = blockIdx.x;
    const long long p0 = unit * pairs_per_unit;
    long long p1 = p0 + pairs_per_unit;
    if (p1 > npairs) p1 = npairs;
    long long pw = (2 * p0 - warm_blocks) / 2;
    if (pw < 0) pw = 0;
    if (p0 >= npairs) pw = p1 = 0;
    for (int i = t; i < FH_N; i += FH_T) {
        acc0[i] = 0.f;
        acc1[i] = 0.f;
    }
    const long long iters = p1 - pw;
    const float sc = 64.0f / (float)FH_N;  // 1/N with H's 2^-6 undone
    __syncthreads();
    for (long long it = 0; it < iters; ++it) {
        const long long p = pw + it;
        const long long b = 2 * p;
        // 32-bit offsets from the pair's first sample: lim0 / lim1 = valid
        // samples of blocks b and b+1
        const long long base = b * hop;
        const float* xb = x + base;
        const int lim0 = fh_count(nx - base, hop), lim1 = fh_count(nx - base - hop, hop);
        V v[FH_E];
#pragma unroll
        for (int m = 0; m < FH_E; ++m) {
            const int i = t + m * FH_T;
            float re = 0.f, im = 0.f;
            if (i < lim0) re = __ldcs(xb + i);
            if (i < lim1) im = __ldcs(xb + hop + i);
            if constexpr (MODE == MFFT_CONV_FP16_PURE) v[m] = __floats2half2_rn(re, im);
            else v[m] = make_float2(re, im);
        }
        hpass<A, 0>(v, t, buf, tw);
        // X and X*H are stored as half2 (fft_fused_convolve_fp16.metal:172-182,
        // 333-341, 482-491); then conj for the inverse through the forward FFT
#pragma unroll
        for (int m = 0; m < FH_E; ++m) {
            const float2 hf = __ldg(H + t + m * FH_T);
            const float2 hs = make_float2(hf.x * FH_HSCALE, hf.y * FH_HSCALE);
            if constexpr (MODE == MFFT_CONV_FP16_STORAGE) {
                v[m] = cconj(round_h(cmul(round_h(v[m]), hs)));
            } else if constexpr (MODE == MFFT_CONV_FP16_MIXED) {
                v[m] = cconj(f2(hcmul(h2(v[m]), h2(hs))));
            } else {
                v[m] = __hmul2(hcmul(v[m], h2(hs)), __floats2half2_rn(1.f, -1.f));
            }
        }
        hpass<A, 0>(v, t, buf, tw);
        // y = conj(v) / N: real part = block b, imaginary part = block b + 1;
        // pure mode scales in FP16 (:141-147)
        auto out = [&](int m) -> float2 {
            if constexpr (MODE == MFFT_CONV_FP16_PURE) return f2(__hmul2(v[m], __floats2half2_rn(sc, -sc)));
            else return make_float2(v[m].x * sc, -v[m].y * sc);
        };
        const bool write = p >= p0;
        float* yb = y + base;
        const int wlim0 = write ? fh_count(ny - base, hop) : 0;
        const int wlim1 = write ? fh_count(ny - base - hop, hop) : 0;
#pragma unroll
        for (int m = 0; m < FH_E; ++m) {
            const int i = t + m * FH_T;
            const float val = out(m).x + acc0[i];
            if (i < hop) {
                if (i < wlim0) __stcs(yb + i, val);
            } else {
                acc1[i - hop] = val;
            }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < FH_E; ++m) {
            const int i = t + m * FH_T;
            const float val = out(m).y + acc1[i];
            if (i < hop) {
                if (i < wlim1) __stcs(yb + hop + i, val);
            } else {
                acc0[i - hop] = val;
            }
        }
        __syncthreads();
    }
}

template <int MODE>
int fh_occ() {
    if (cudaFuncSetAttribute(k_conv_fwd_h<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, FH_SMEM) != cudaSuccess)
        return 0;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_conv_fwd_h<MODE>, FH_T, FH_SMEM) != cudaSuccess) return 0;
    return occ;
}

}  // namespace

int conv_fp16_ctas_per_sm(int mode) {
    switch (mode) {
        case MFFT_CONV_FP16_STORAGE: return fh_occ<MFFT_CONV_FP16_STORAGE>();
        case MFFT_CONV_FP16_MIXED: return fh_occ<MFFT_CONV_FP16_MIXED>();
        case MFFT_CONV_FP16_PURE: return fh_occ<MFFT_CONV_FP16_PURE>();
        default: return 0;
    }
}

cudaError_t conv_fp16_forward(int mode, long long ctas, cudaStream_t s, const float* x, long long nx, float* y,
                              long long ny, const float2* H, const float2* tw, int hop, long long npairs,
                              long long ppu, int warm) {
    const dim3 grid((unsigned)ctas);
    switch (mode) {
        case MFFT_CONV_FP16_STORAGE:
            k_conv_fwd_h<MFFT_CONV_FP16_STORAGE><<<grid, FH_T, FH_SMEM, s>>>(x, nx, y, ny, H, tw, hop, npairs, ppu, warm);
            break;
        case MFFT_CONV_FP16_MIXED:
            k_conv_fwd_h<MFFT_CONV_FP16_MIXED><<<grid, FH_T, FH_SMEM, s>>>(x, nx, y, ny, H, tw, hop, npairs, ppu, warm);
            break;
        case MFFT_CONV_FP16_PURE:
            k_conv_fwd_h<MFFT_CONV_FP16_PURE><<<grid, FH_T, FH_SMEM, s>>>(x, nx, y, ny, H, tw, hop, npairs, ppu, warm);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace mfft
