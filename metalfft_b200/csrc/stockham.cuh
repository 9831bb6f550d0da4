// stockham.cuh -- the in-register / in-shared-memory Stockham FFT used by
// every kernel of libmfft that transforms a whole line on chip.
//
// fft_regs<N, E, WS>(v, t, buf, tw):
//   on entry  v[m] = x[t + m*T]   (T = N/E threads cooperate on one line)
//   on return v[m] = X[t + m*T]   (natural order, forward sign, unscaled)
// buf maps a line index i in [0, N) to the shared-memory slot of the line's
// exchange area (PadLine: one line per area; ColLine / SwzLine: C lines
// interleaved so that threads of different lines sit on different banks);
// tw the line's twiddle rows (SPlan<N,E>::TWSIZE float2, built by
// gen_twiddles on the device in FP64).  WS: the T threads of a line sit in
// one warp, so __syncwarp orders the exchange; otherwise __syncthreads.
//
// It is the radix-E restatement of the reference's passes
// (Sources/MetalFFT/Resources/fft_multisize.metal:62-687: load
// buf[tid + r*T], twiddle by position within the span, butterfly, write to
// grp*stride*R + pos + r*stride) with E = 16 by default: N = 4096 takes 3
// passes and 2 exchanges instead of the reference's 6 radix-4 passes, and the
// first and last passes read and write global memory directly with
// consecutive threads on consecutive elements.
#pragma once

#include "fft_common.cuh"

namespace mfft {

template <bool WS>
__device__ __forceinline__ void line_sync() {
    if constexpr (WS) __syncwarp();
    else __syncthreads();
}

// One line per padded area.
struct PadLine {
    float2* base;
    __device__ __forceinline__ float2& operator[](int i) const { return base[spad(i)]; }
};
// The same layout, declared splittable: kPadStride says the layout is
// base + spad(i) * kPadStride, so the passes address it as
// at(a)[spad(b) * kPadStride] wherever spad(a + b) = spad(a) + spad(b) (b a
// multiple of 16, or a a multiple of 16 and b < 16): one address computation
// per group of R writes and one per thread for the reads, the rest constant
// offsets.  Kept apart from PadLine because the split is not a gain in every
// kernel (the real-input FFT measured slower with it).
struct PadLineS {
    float2* base;
    static constexpr int kPadStride = 1;
    __device__ __forceinline__ float2& operator[](int i) const { return base[spad(i)]; }
    __device__ __forceinline__ float2* at(int i) const { return base + spad(i); }
};
// kPadStride of a layout, 0 for layouts without one.
template <class Buf>
__host__ __device__ constexpr auto pad_stride_of(int) -> decltype(Buf::kPadStride) {
    return Buf::kPadStride;
}
template <class Buf>
__host__ __device__ constexpr int pad_stride_of(long) {
    return 0;
}
// C lines interleaved element by element: line c, element i at i*C + c.
template <int C>
struct ColLine {
    float2* base;
    int c;
    __device__ __forceinline__ float2& operator[](int i) const { return base[i * C + c]; }
};
// C lines interleaved element by element over the padded index: line c,
// element i at spad(i)*C + c (splittable, kPadStride = C).  With C = 2 or 4
// and radix-16 passes, the first pass's writes (elements 16j + r, j = the
// thread) land 16*C float2 apart, all on one bank, in ColLine; the pad puts
// consecutive threads 17*C float2 apart, on different banks, while the reads
// (consecutive i) and the later passes' writes (consecutive i within a
// 16-element group) stay conflict-free.
template <int C>
struct ColPadLine {
    float2* base;
    int c;
    static constexpr int kPadStride = C;
    __device__ __forceinline__ float2& operator[](int i) const { return base[spad(i) * C + c]; }
    __device__ __forceinline__ float2* at(int i) const { return base + spad(i) * C + c; }
};
// C lines interleaved with an XOR swizzle, so that both a warp walking one
// line (i consecutive, c fixed) and a warp walking across lines (c
// consecutive, i fixed) hit distinct banks: line c, element i at
// i*C + (c ^ (i mod C)).
template <int C>
struct SwzLine {
    float2* base;
    int c;
    __device__ __forceinline__ float2& operator[](int i) const { return base[i * C + (c ^ (i & (C - 1)))]; }
};

template <int N, int E, int P, bool WS>
struct StockhamPass {
    template <class Buf>
    static __device__ __forceinline__ void run(float2 (&v)[E], int t, const Buf& buf,
                                               const float2* __restrict__ tw) {
        using PL = SPlan<N, E>;
        constexpr int R = PL::radix(P);
        constexpr int NS = PL::span(P);
        constexpr int B = E / R;
        constexpr int T = PL::T;
        // padded layouts: one address per group of R writes (and per thread for the
        // reads), the rest constant offsets, where the split is exact
        constexpr int S = pad_stride_of<Buf>(0);
        constexpr bool WSPLIT = S > 0 && (NS % 16 == 0 || (NS == 1 && R == 16));
        constexpr bool RSPLIT = S > 0 && T % 16 == 0;
        if constexpr (NS > 1) {
#pragma unroll
            for (int b = 0; b < B; ++b) {
                const int k = (t + b * T) & (NS - 1);
                apply_twiddles<R, B>(v + b, tw + PL::twoff(P) + k * PL::twrow(R));
            }
        }
#pragma unroll
        for (int b = 0; b < B; ++b) dft<R, B>(v + b);
        if constexpr (P + 1 < PL::NPASS) {
#pragma unroll
            for (int b = 0; b < B; ++b) {
                const int j = t + b * T;
                const int k = j & (NS - 1);
                const int d = (j - k) * R + k;
                if constexpr (WSPLIT) {
                    float2* p = buf.at(d);
#pragma unroll
                    for (int r = 0; r < R; ++r) p[spad(r * NS) * S] = v[b + r * B];
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r) buf[d + r * NS] = v[b + r * B];
                }
            }
            line_sync<WS>();
            if constexpr (RSPLIT) {
                const float2* p = buf.at(t);
#pragma unroll
                for (int m = 0; m < E; ++m) v[m] = p[spad(m * T) * S];
            } else {
#pragma unroll
                for (int m = 0; m < E; ++m) v[m] = buf[t + m * T];
            }
            line_sync<WS>();
            StockhamPass<N, E, P + 1, WS>::run(v, t, buf, tw);
        }
    }
};

template <int N, int E, bool WS, class Buf>
__device__ __forceinline__ void fft_regs(float2 (&v)[E], int t, const Buf& buf,
                                         const float2* __restrict__ tw) {
    StockhamPass<N, E, 0, WS>::run(v, t, buf, tw);
}

// Twiddle rows of pass p: row k holds e^{-2*pi*i*e*k/(Ns*R)} for e = 1, 2, 4, 8
// (first `rowlen` of them), in FP64 (sincospi) rounded once to FP32.
__global__ void k_twiddle_rows(float2* tw, int off, int ns, int radix, int rowlen);

template <int N, int E>
inline void gen_twiddles(float2* tw, cudaStream_t s) {
    using PL = SPlan<N, E>;
    for (int p = 1; p < PL::NPASS; ++p) {
        int cnt = PL::span(p) * PL::twrow(PL::radix(p));
        k_twiddle_rows<<<(cnt + 255) / 256, 256, 0, s>>>(tw, PL::twoff(p), PL::span(p), PL::radix(p),
                                                          PL::twrow(PL::radix(p)));
    }
}

}  // namespace mfft
