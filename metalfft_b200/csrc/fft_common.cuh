// fft_common.cuh -- complex arithmetic, radix-2/4/8/16 butterflies and the
// compile-time Stockham plan shared by every FFT kernel of libmfft.
//
// Sign convention: forward kernels compute X[k] = sum_j x[j] e^{-2*pi*i*j*k/N}
// (Sources/MetalFFT/Resources/fft_multisize.metal:70, TWO_PI_OVER_N = -2*pi/N).
// Inverse transforms are formed as (1/N) conj(FFT(conj(X))) by the callers
// (Sources/MetalFFT/FFT/MetalFFT.swift:56-65), fused into their loads/stores.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mfft {

__host__ __device__ constexpr int ilog2c(long long n) {
    int l = 0;
    while ((1LL << l) < n) ++l;
    return l;
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// -i * a
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }
// e^{-i*pi/4} * a = ((a.x + a.y), (a.y - a.x)) / sqrt(2)
__device__ __forceinline__ float2 mul_w8_1(float2 a) {
    const float r = 0.70710678118654752440f;
    return make_float2((a.x + a.y) * r, (a.y - a.x) * r);
}
// e^{-3i*pi/4} * a = ((a.y - a.x), -(a.x + a.y)) / sqrt(2)
__device__ __forceinline__ float2 mul_w8_3(float2 a) {
    const float r = 0.70710678118654752440f;
    return make_float2((a.y - a.x) * r, -(a.x + a.y) * r);
}
// (wr + i*wi) * a for compile-time constants
__device__ __forceinline__ float2 mul_c(float2 a, float wr, float wi) {
    return make_float2(fmaf(a.x, wr, -a.y * wi), fmaf(a.x, wi, a.y * wr));
}

// ---- butterflies on v[0], v[S], v[2S], ... (forward sign), in place,
// ---- natural order in and out.

template <int S>
__device__ __forceinline__ void dft2(float2* v) {
    float2 a = v[0], b = v[S];
    v[0] = cadd(a, b);
    v[S] = csub(a, b);
}

template <int S>
__device__ __forceinline__ void dft4(float2* v) {
    float2 t0 = cadd(v[0], v[2 * S]);
    float2 t1 = csub(v[0], v[2 * S]);
    float2 t2 = cadd(v[S], v[3 * S]);
    float2 t3 = mul_mi(csub(v[S], v[3 * S]));
    v[0] = cadd(t0, t2);
    v[2 * S] = csub(t0, t2);
    v[S] = cadd(t1, t3);
    v[3 * S] = csub(t1, t3);
}

// 8-point DFT as two 4-point DFTs (even / odd samples) and one radix-2 layer.
template <int S>
__device__ __forceinline__ void dft8(float2* v) {
    float2 a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = v[i * S];
    dft4<2>(a);      // E_k at a[0], a[2], a[4], a[6]
    dft4<2>(a + 1);  // O_k at a[1], a[3], a[5], a[7]
    a[3] = mul_w8_1(a[3]);
    a[5] = mul_mi(a[5]);
    a[7] = mul_w8_3(a[7]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k * S] = cadd(a[2 * k], a[2 * k + 1]);
        v[(k + 4) * S] = csub(a[2 * k], a[2 * k + 1]);
    }
}

// 16-point DFT as 4 x 4: n = 4*n1 + n2, k = k1 + 4*k2.
template <int S>
__device__ __forceinline__ void dft16(float2* v) {
    const float C = 0.92387953251128675613f;  // cos(pi/8)
    const float D = 0.38268343236508977173f;  // sin(pi/8)
    float2 a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = v[i * S];
    // 4-point DFTs over n1 for each n2: elements a[n2 + 4*n1] -> A[n2][k1] at a[n2 + 4*k1]
    dft4<4>(a + 0);
    dft4<4>(a + 1);
    dft4<4>(a + 2);
    dft4<4>(a + 3);
    // twiddles W16^(n2*k1) at a[n2 + 4*k1]
    a[5] = mul_c(a[5], C, -D);    // n2=1,k1=1: W^1
    a[9] = mul_w8_1(a[9]);        // n2=1,k1=2: W^2
    a[13] = mul_c(a[13], D, -C);  // n2=1,k1=3: W^3
    a[6] = mul_w8_1(a[6]);        // n2=2,k1=1: W^2
    a[10] = mul_mi(a[10]);        // n2=2,k1=2: W^4
    a[14] = mul_w8_3(a[14]);      // n2=2,k1=3: W^6
    a[7] = mul_c(a[7], D, -C);    // n2=3,k1=1: W^3
    a[11] = mul_w8_3(a[11]);      // n2=3,k1=2: W^6
    a[15] = mul_c(a[15], -C, D);  // n2=3,k1=3: W^9
    // 4-point DFTs over n2 for each k1: elements a[4*k1 + n2] -> X[k1 + 4*k2] at a[4*k1 + k2]
    dft4<1>(a + 0);
    dft4<1>(a + 4);
    dft4<1>(a + 8);
    dft4<1>(a + 12);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[(k1 + 4 * k2) * S] = a[4 * k1 + k2];
}

template <int R, int S>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) dft2<S>(v);
    else if constexpr (R == 4) dft4<S>(v);
    else if constexpr (R == 8) dft8<S>(v);
    else if constexpr (R == 16) dft16<S>(v);
}

// Compile-time Stockham plan for a length-N transform held E elements per
// thread: passes of radix E, then one tail pass of radix 2^(log2 N mod log2 E)
// (the reference places its radix-2 pass last as well:
// fft_multisize.metal:252-280).  Pass p has span Ns(p) = prod of earlier
// radices; thread t loads elements t + m*T (T = N/E) in every pass, applies
// twiddles e^{-2*pi*i*r*k/(Ns*R)} (k = j mod Ns) and writes element r of
// butterfly j to expand(j) + r*Ns, expand(j) = (j/Ns)*Ns*R + (j mod Ns).
template <int N, int E>
struct SPlan {
    static constexpr int LN = ilog2c(N);
    static constexpr int LE = ilog2c(E);
    static constexpr int NFULL = LN / LE;
    static constexpr int REM = LN % LE;
    static constexpr int NPASS = NFULL + (REM ? 1 : 0);
    static constexpr int T = N / E;
    __host__ __device__ static constexpr int radix(int p) { return p < NFULL ? E : (1 << REM); }
    __host__ __device__ static constexpr int span(int p) {
        int s = 1;
        for (int q = 0; q < p; ++q) s *= radix(q);
        return s;
    }
    // float2 per twiddle row: {w1, w2, w4, w8} for radix 8/16, {w1, w2} below
    __host__ __device__ static constexpr int twrow(int r) { return r >= 8 ? 4 : 2; }
    // offset (in float2) of pass p's twiddle rows (k = 0 .. Ns-1)
    __host__ __device__ static constexpr int twoff(int p) {
        int o = 0;
        for (int q = 1; q < p; ++q) o += span(q) * twrow(radix(q));
        return o;
    }
    static constexpr int TWSIZE = twoff(NPASS) > 0 ? twoff(NPASS) : 2;
};

// Multiplies v[r*B] (r = 1 .. R-1) by w^r, w = e^{-2*pi*i*k/(Ns*R)}, from the
// row {w, w^2, w^4, w^8}: the other powers are products of at most three
// table values (w^15 = ((w * w^2) * w^4) * w^8), so every twiddle stays within
// a few ulp while a thread reads 16 or 32 bytes per pass instead of 8*R.
template <int R, int B>
__device__ __forceinline__ void apply_twiddles(float2* v, const float2* __restrict__ row) {
    const float4 q0 = __ldg(reinterpret_cast<const float4*>(row));
    const float2 w1 = make_float2(q0.x, q0.y);
    const float2 w2 = make_float2(q0.z, q0.w);
    if constexpr (R == 2) {
        v[B] = cmul(v[B], w1);
    } else if constexpr (R == 4) {
        v[B] = cmul(v[B], w1);
        v[2 * B] = cmul(v[2 * B], w2);
        v[3 * B] = cmul(v[3 * B], cmul(w1, w2));
    } else {
        const float4 q1 = __ldg(reinterpret_cast<const float4*>(row) + 1);
        const float2 w4 = make_float2(q1.x, q1.y);
        const float2 w3 = cmul(w1, w2);
        const float2 w5 = cmul(w1, w4);
        const float2 w6 = cmul(w2, w4);
        const float2 w7 = cmul(w3, w4);
        v[B] = cmul(v[B], w1);
        v[2 * B] = cmul(v[2 * B], w2);
        v[3 * B] = cmul(v[3 * B], w3);
        v[4 * B] = cmul(v[4 * B], w4);
        v[5 * B] = cmul(v[5 * B], w5);
        v[6 * B] = cmul(v[6 * B], w6);
        v[7 * B] = cmul(v[7 * B], w7);
        if constexpr (R == 16) {
            const float2 w8 = make_float2(q1.z, q1.w);
            v[8 * B] = cmul(v[8 * B], w8);
            v[9 * B] = cmul(v[9 * B], cmul(w1, w8));
            v[10 * B] = cmul(v[10 * B], cmul(w2, w8));
            v[11 * B] = cmul(v[11 * B], cmul(w3, w8));
            v[12 * B] = cmul(v[12 * B], cmul(w4, w8));
            v[13 * B] = cmul(v[13 * B], cmul(w5, w8));
            v[14 * B] = cmul(v[14 * B], cmul(w6, w8));
            v[15 * B] = cmul(v[15 * B], cmul(w7, w8));
        }
    }
}

// Padded shared-memory index: one spare float2 per 16 keeps the Stockham
// write patterns (stride R*Ns) free of bank conflicts.
__device__ __forceinline__ int spad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int spad_size(int n) { return n + n / 16; }

}  // namespace mfft
