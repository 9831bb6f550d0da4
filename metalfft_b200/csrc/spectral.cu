// spectral.cu -- STFT, Welch power spectral density and magnitude-squared
// coherence as batched single launches.
//
// Reference: STFT.analyze (Sources/MetalFFT/DSP/STFT.swift:79-108),
// PSD.welch (DSP/PSD.swift:18-58) and PSD.coherence (DSP/PSD.swift:71-134)
// loop over frames on the host: per frame a vDSP window multiply, a complex
// pack with zero imaginary part, one GPU forward FFT of fftSize points and a
// CPU accumulation.  Here every frame of the signal is transformed in one
// launch:
//  * two real frames travel as the real and imaginary parts of one complex
//    line (STFT and Welch: frames 2p and 2p+1; coherence: frame f of a and of
//    b); the Hermitian split A_k = (Z_k + conj Z_{n-k})/2,
//    B_k = (Z_k - conj Z_{n-k})/(2i) recovers both spectra, so a pair of
//    frames costs one transform instead of two;
//  * the window multiply is fused into the load (each thread keeps its 16
//    window values in registers across frames);
//  * Welch and coherence sums accumulate per bin in shared memory (global
//    memory when it does not fit, coherence at 16384) owned by one thread per
//    bin, are written per walker and summed over walkers in a fixed order,
//    then normalised: deterministic, no atomics.
//
// PSD.crossSpectral (DSP/CrossSpectral.swift:56-152) also loops per frame:
// a multi-channel FFT, a per-bin kernel for |X_c|^2, X_i conj(X_j) and the
// per-frame coherence (Resources/fft_cross_spectral.metal:29-63), then CPU
// sums.  Here the frames go through in chunks small enough for their spectra
// to stay in L2:
//  * k_xstft transforms frame pairs of every channel of the chunk (the same
//    two-real-frames-per-line split) and keeps bins 0 .. n/2 - 1 (real
//    input: X_{n-k} = conj X_k); the real Nyquist bin of every frame goes to
//    a side array for the whole call, summed by k_xspec_nyq;
//  * k_xspec_acc owns a tile of bins and a slice of the chunk's frames; its
//    warp groups split the upper-triangle channel pairs, with the pair sums in
//    registers and the channel values of a few frames staged in shared memory
//    by cp.async; the sums of each frame slice carry over from chunk to chunk
//    in a fixed order.  For 2, 4 and 8 channels the channel count is a
//    compile-time constant: each thread loads a bin's C values and powers
//    into registers once per frame and forms its pairs from them with static
//    indices; other counts read each pair's two values through a table of
//    byte offsets;
//  * k_xspec_finish sums the slices in FP64, divides by the frame count and
//    mirrors bins n/2+1 .. n-1 from their conjugates.
#include <vector>

#include "capi_internal.h"
#include "pdl.cuh"
#include "stockham.cuh"

namespace mfft {

namespace {

constexpr int SP_E = 16;

template <int FFT>
struct SpGeom {
    static constexpr int T = FFT / SP_E;
    static constexpr int LINES = T >= 128 ? 1 : 128 / T;  // lines (walkers) per CTA
    static constexpr int THREADS = T * LINES;
    static constexpr bool WS = (T <= 32);
    static constexpr int XCH = LINES * spad_size(FFT);  // exchange area, float2
    // accumulation kernels: up to three CTAs of <= 256 threads per SM (80
    // registers at fft 4096, no spills)
    static constexpr int MINB = THREADS <= 256 ? 3 : 1;
    // per-line accumulator planes: Welch 1 (power), coherence 4 (Sxx, Syy, Re, Im Sxy)
    template <int PLANES>
    static constexpr bool acc_smem() {
        return XCH * 8 + LINES * PLANES * FFT * 4 <= 227 * 1024;
    }
    template <int PLANES>
    static constexpr int smem_bytes() {
        return XCH * 8 + (acc_smem<PLANES>() ? LINES * PLANES * FFT * 4 : 0);
    }
};

// Z (natural order in v, thread t holds k = t + m*T) -> A, B spectra of the
// real and imaginary inputs, handed bin by bin to use(m, A, B) so that no
// second and third spectrum array is kept in registers; Z_{n-k} comes
// through the exchange area.
template <int FFT, bool WS, class Buf, class Use>
__device__ __forceinline__ void hermitian_split(const float2 (&v)[SP_E], int t, const Buf& buf, Use&& use) {
    constexpr int T = FFT / SP_E;
#pragma unroll
    for (int m = 0; m < SP_E; ++m) buf[t + m * T] = v[m];
    line_sync<WS>();
#pragma unroll
    for (int m = 0; m < SP_E; ++m) {
        const int k = t + m * T;
        const float2 zc = cconj(buf[(FFT - k) & (FFT - 1)]);
        const float2 A = make_float2(0.5f * (v[m].x + zc.x), 0.5f * (v[m].y + zc.y));
        const float2 d = make_float2(0.5f * (v[m].x - zc.x), 0.5f * (v[m].y - zc.y));
        use(m, A, make_float2(d.y, -d.x));  // B = d / i
    }
    line_sync<WS>();
}

// frames (2p, 2p+1) of x, windowed, as one complex line
template <int FFT>
__device__ __forceinline__ void load_pair(const float* __restrict__ x, long long frames, int hop, long long p, int t,
                                          const float (&w)[SP_E], float2 (&v)[SP_E]) {
    constexpr int T = FFT / SP_E;
    const long long f0 = 2 * p;
    const bool ok0 = f0 < frames, ok1 = f0 + 1 < frames;
    const float* x0 = x + f0 * hop + t;
#pragma unroll
    for (int m = 0; m < SP_E; ++m) {
        const float re = ok0 ? __ldcs(x0 + m * T) * w[m] : 0.f;
        const float im = ok1 ? __ldcs(x0 + hop + m * T) * w[m] : 0.f;
        v[m] = make_float2(re, im);
    }
}

template <int FFT>
__global__ void __launch_bounds__(SpGeom<FFT>::THREADS)
    k_stft(const float* __restrict__ x, long long frames, int hop, const float* __restrict__ win,
           const float2* __restrict__ tw, float2* __restrict__ spec, float* __restrict__ power) {
    using G = SpGeom<FFT>;
    constexpr int T = G::T;
    extern __shared__ __align__(16) float2 smem[];
    const int lf = threadIdx.x / T, t = threadIdx.x % T;
    const PadLine buf{smem + lf * spad_size(FFT)};
    const long long p = (long long)blockIdx.x * G::LINES + lf;  // frame pair (idle lines still sync)
    float w[SP_E];
#pragma unroll
    for (int m = 0; m < SP_E; ++m) w[m] = __ldg(win + t + m * T);
    float2 v[SP_E];
    load_pair<FFT>(x, frames, hop, p, t, w, v);
    fft_regs<FFT, SP_E, G::WS>(v, t, buf, tw);
    const long long f0 = 2 * p;
    const bool ok0 = f0 < frames, ok1 = f0 + 1 < frames;
    float2* s0 = spec ? spec + f0 * FFT + t : nullptr;
    float* p0 = power ? power + f0 * FFT + t : nullptr;
    hermitian_split<FFT, G::WS>(v, t, buf, [&](int m, float2 A, float2 B) {
        if (s0) {
            if (ok0) __stcs(s0 + m * T, A);
            if (ok1) __stcs(s0 + FFT + m * T, B);
        }
        if (p0) {
            if (ok0) __stcs(p0 + m * T, A.x * A.x + A.y * A.y);
            if (ok1) __stcs(p0 + FFT + m * T, B.x * B.x + B.y * B.y);
        }
    });
}

// Welch (COH = false): walker u owns frame pairs [u*per, (u+1)*per) of x and
// sums |A|^2 + |B|^2 per bin.  Coherence (COH = true): walker u owns frames
// [u*per, (u+1)*per); line = frame f of a (re) and of b (im); sums |A|^2,
// |B|^2, Re and Im of A conj(B).  Sums land in part[u][plane][FFT].
template <int FFT, bool COH>
__global__ void __launch_bounds__(SpGeom<FFT>::THREADS, SpGeom<FFT>::MINB)
    k_spec_acc(const float* __restrict__ a, const float* __restrict__ b, long long frames, int hop,
               const float* __restrict__ win, const float2* __restrict__ tw, long long work, long long per,
               float* __restrict__ part) {
    using G = SpGeom<FFT>;
    constexpr int T = G::T;
    constexpr int PLANES = COH ? 4 : 1;
    constexpr bool ACC_SMEM = G::template acc_smem<PLANES>();
    extern __shared__ __align__(16) float2 smem[];
    const int lf = threadIdx.x / T, t = threadIdx.x % T;
    const PadLineS buf{smem + lf * spad_size(FFT)};
    const long long u = (long long)blockIdx.x * G::LINES + lf;
    float* acc = ACC_SMEM ? reinterpret_cast<float*>(smem + G::XCH) + lf * PLANES * FFT : part + u * PLANES * FFT;
#pragma unroll
    for (int pl = 0; pl < PLANES; ++pl)
#pragma unroll
        for (int m = 0; m < SP_E; ++m) acc[pl * FFT + t + m * T] = 0.f;
    float w[SP_E];
#pragma unroll
    for (int m = 0; m < SP_E; ++m) w[m] = __ldg(win + t + m * T);
    const long long i0 = u * per;
    for (long long it = 0; it < per; ++it) {  // same count on every line of the CTA
        const long long i = i0 + it;
        const bool active = i < work;
        float2 v[SP_E];
        if constexpr (COH) {
            const float* pa = a + i * hop + t;
            const float* pb = b + i * hop + t;
#pragma unroll
            for (int m = 0; m < SP_E; ++m)
                v[m] = active ? make_float2(__ldcs(pa + m * T) * w[m], __ldcs(pb + m * T) * w[m]) : make_float2(0.f, 0.f);
        } else {
            load_pair<FFT>(a, active ? frames : 0, hop, i, t, w, v);
        }
        fft_regs<FFT, SP_E, G::WS>(v, t, buf, tw);
        if constexpr (COH) {
            // bins 0 .. n/2 only: for real frames A_{n-k} and B_{n-k} are the
            // exact conjugates of A_k and B_k, so the sums at n - k mirror
            // these (k_spec_finish reads them there)
            hermitian_split<FFT, G::WS>(v, t, buf, [&](int m, float2 A, float2 B) {
                const int k = t + m * T;
                if (k <= FFT / 2) {
                    acc[k] += A.x * A.x + A.y * A.y;
                    acc[FFT + k] += B.x * B.x + B.y * B.y;
                    acc[2 * FFT + k] += A.x * B.x + A.y * B.y;
                    acc[3 * FFT + k] += A.y * B.x - A.x * B.y;
                }
            });
        } else {
            // |A_k|^2 + |B_k|^2 = (|Z_k|^2 + |Z_{n-k}|^2) / 2 for A, B the spectra
            // of the real and imaginary inputs: sum |Z_k|^2 here, fold k and n-k
            // once per walker below (no Hermitian split per line; a missing
            // frame 2i+1 leaves Z Hermitian and the fold gives |A_k|^2)
#pragma unroll
            for (int m = 0; m < SP_E; ++m) acc[t + m * T] += v[m].x * v[m].x + v[m].y * v[m].y;
        }
    }
    if constexpr (!COH) {
        __syncthreads();  // every thread's sums are written
        float fold[SP_E];
#pragma unroll
        for (int m = 0; m < SP_E; ++m) {
            const int k = t + m * T;
            fold[m] = 0.5f * (acc[k] + acc[(FFT - k) & (FFT - 1)]);
        }
        __syncthreads();  // every read of the unfolded sums is done
#pragma unroll
        for (int m = 0; m < SP_E; ++m) acc[t + m * T] = fold[m];
        if constexpr (ACC_SMEM) __syncthreads();
    }
    if constexpr (ACC_SMEM) {
        float* dst = part + u * PLANES * FFT;
#pragma unroll
        for (int pl = 0; pl < PLANES; ++pl)
#pragma unroll
            for (int m = 0; m < SP_E; ++m) dst[pl * FFT + t + m * T] = acc[pl * FFT + t + m * T];
    }
}

// Sum over walkers, then the normalisation.  A CTA owns 16 consecutive bins;
// thread (run r, bin b) sums walkers [r*R, (r+1)*R) of its bin in walker order
// (FP64), and lane b then adds the 16 runs in run order: a fixed order, with
// fft/16 CTAs instead of one serial thread per bin.
constexpr int FIN_BINS = 16, FIN_RUNS = 16;
template <bool COH>
__global__ void __launch_bounds__(FIN_BINS * FIN_RUNS)
    k_spec_finish(const float* __restrict__ part, long long units, int fft, float scale, float* __restrict__ out) {
    constexpr int PLANES = COH ? 4 : 1;
    __shared__ double red[FIN_RUNS][PLANES][FIN_BINS];
    const int b = threadIdx.x % FIN_BINS, r = threadIdx.x / FIN_BINS;
    const int k = blockIdx.x * FIN_BINS + b;  // fft is a multiple of FIN_BINS
    // coherence sums exist for bins 0 .. n/2; bin k > n/2 has those of n - k
    // (|Sxy|^2, Sxx and Syy are symmetric)
    const int ks = (COH && k > fft / 2) ? fft - k : k;
    const long long run = (units + FIN_RUNS - 1) / FIN_RUNS, u0 = r * run;
    const long long u1 = u0 + run < units ? u0 + run : units;
    double s[PLANES];
#pragma unroll
    for (int pl = 0; pl < PLANES; ++pl) s[pl] = 0.0;
    for (long long u = u0; u < u1; ++u)
#pragma unroll
        for (int pl = 0; pl < PLANES; ++pl) s[pl] += part[(u * PLANES + pl) * fft + ks];
#pragma unroll
    for (int pl = 0; pl < PLANES; ++pl) red[r][pl][b] = s[pl];
    __syncthreads();
    if (r != 0) return;
#pragma unroll
    for (int pl = 0; pl < PLANES; ++pl) {
        double tot = 0.0;
        for (int q = 0; q < FIN_RUNS; ++q) tot += red[q][pl][b];
        s[pl] = tot;
    }
    if constexpr (COH) {
        const double den = s[0] * s[1];
        out[k] = den > 0.0 ? (float)((s[2] * s[2] + s[3] * s[3]) / den) : 0.f;
    } else {
        out[k] = (float)(s[0] * scale);
    }
}

// ---- cross-spectral -----------------------------------------------------

// spectra of a chunk: X[(f * C + c) * hs + k], k = 0 .. n/2, hs = n/2 + 16
// (rows stay 128-byte aligned)
__host__ __device__ constexpr int xs_stride(int fft) { return fft / 2 + 16; }

template <int FFT>
__global__ void __launch_bounds__(SpGeom<FFT>::THREADS)
    k_xstft(const float* __restrict__ x, long long len, int C, long long f0, long long nf, int hop,
            const float* __restrict__ win, const float2* __restrict__ tw, float2* __restrict__ X,
            float* __restrict__ nyq) {
    using G = SpGeom<FFT>;
    constexpr int T = G::T, HS = xs_stride(FFT);
    extern __shared__ __align__(16) float2 smem[];
    // launched as a dependent of the previous chunk's pair kernel, which still
    // reads X: wait for it before any global access
    grid_dep_wait();
    const int lf = threadIdx.x / T, t = threadIdx.x % T;
    const PadLine buf{smem + lf * spad_size(FFT)};
    const long long pairs = (nf + 1) / 2;
    const long long l = (long long)blockIdx.x * G::LINES + lf;
    const bool line_ok = l < (long long)C * pairs;  // idle lines still take part in the syncs
    const int c = line_ok ? (int)(l / pairs) : 0;
    const long long p = line_ok ? l - (long long)c * pairs : 0;
    float w[SP_E];
#pragma unroll
    for (int m = 0; m < SP_E; ++m) w[m] = __ldg(win + t + m * T);
    float2 v[SP_E];
    load_pair<FFT>(x + (long long)c * len + f0 * hop, line_ok ? nf : 0, hop, p, t, w, v);
    fft_regs<FFT, SP_E, G::WS>(v, t, buf, tw);
    const bool ok0 = line_ok && 2 * p < nf, ok1 = line_ok && 2 * p + 1 < nf;
    float2* r0 = X + (2 * p * C + c) * HS;
    float2* r1 = r0 + (long long)C * HS;
    // bins 0 .. n/2 - 1 to the chunk's spectra; the Nyquist bin (real for a
    // real frame: A and B at k = n/2 have zero imaginary parts) to nyq[frame][channel]
    // of the whole call
    float* nq = nyq + (f0 + 2 * p) * C + c;
    hermitian_split<FFT, G::WS>(v, t, buf, [&](int m, float2 A, float2 B) {
        const int k = t + m * T;
        if (k == FFT / 2) {
            if (ok0) nq[0] = A.x;
            if (ok1) nq[C] = B.x;
        } else if (k < FFT / 2) {
            if (ok0) r0[k] = A;
            if (ok1) r1[k] = B;
        }
    });
}

// k_xspec_acc geometry: G warp groups split the pairs; KB = XS_THREADS / G
// bins per CTA; up to XQ pairs and xs_pmax(G) channel powers per thread; XF
// frames per stage, XS_ST stage buffers (XS_ST - 1 stages in flight while one
// is summed; <= 98 KB per CTA at any channel count, two CTAs per SM).
constexpr int XS_THREADS = 512, XQ = 8, XF = 2, XS_ST = 3, XS_MAX_CH = 16, XS_MAX_G = 16;
constexpr int XS_MAX_PAIRS = XS_MAX_CH * (XS_MAX_CH - 1) / 2;
// largest channel count with ceil(P / G) <= XQ, divided over G groups
__host__ __device__ constexpr int xs_pmax(int g) { return g == 1 ? 4 : g == 2 ? 3 : g <= 8 ? 2 : 1; }
// smallest G in {1, 2, 4, 8, 16} with ceil(P / G) <= XQ
inline int xs_groups(int C) {
    const int P = C * (C - 1) / 2;
    for (int g = 1; g < XS_MAX_G; g *= 2)
        if ((P + g - 1) / g <= XQ) return g;
    return XS_MAX_G;
}
inline int xs_smem(int C, int g) { return XS_ST * XF * C * (XS_THREADS / g) * (int)sizeof(float2); }

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit_xs() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// all but the XS_ST - 1 most recent copy groups have landed
__device__ __forceinline__ void cp_async_wait_xs() {
    asm volatile("cp.async.wait_group %0;" ::"n"(XS_ST - 1) : "memory");
}
// 1/x within one unit in the last place (PTX rcp.approx.f32)
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Upper-triangle pair q of C channels: (xs_pi, xs_pj), row i holding the
// C - 1 - i pairs (i, i+1) .. (i, C-1) (fft_cross_spectral.metal:51-61 order).
__host__ __device__ constexpr int xs_pi(int C, int q) {
    int i = 0;
    while (q >= C - 1 - i) q -= C - 1 - i++;
    return i;
}
__host__ __device__ constexpr int xs_pj(int C, int q) {
    int i = 0;
    while (q >= C - 1 - i) q -= C - 1 - i++;
    return i + 1 + q;
}

// One frame of one bin for warp group GI when the channel count C is a
// compile-time constant: the C channel values and powers sit in registers
// (loaded and squared once per bin and frame, as the reference's kernel does),
// and every pair of the group reads them with static indices.
template <int C, int G, int GI, bool COH, int Q, int QEND>
struct XsPairs {
    static __device__ __forceinline__ void run(const float2 (&u)[C], const float (&p)[C], float (&cr)[XQ],
                                               float (&ci)[XQ], float (&ch)[XQ]) {
        if constexpr (Q < QEND) {
            constexpr int P = C * (C - 1) / 2, q0 = GI * ((P + G - 1) / G);
            constexpr int i = xs_pi(C, q0 + Q), j = xs_pj(C, q0 + Q);
            // S_ij = X_i conj(X_j) (fft_cross_spectral.metal:57-58)
            const float sr = u[i].x * u[j].x + u[i].y * u[j].y;
            const float sim = u[i].y * u[j].x - u[i].x * u[j].y;
            cr[Q] += sr;
            ci[Q] += sim;
            if constexpr (COH) ch[Q] += (sr * sr + sim * sim) * rcp_approx(fmaxf(p[i] * p[j], 1e-30f));
            XsPairs<C, G, GI, COH, Q + 1, QEND>::run(u, p, cr, ci, ch);
        }
    }
};

template <int C, int G, int GI, bool COH>
__device__ __forceinline__ void xs_frame_static(const float2* U, int KB, float (&pw)[xs_pmax(G)], float (&cr)[XQ],
                                                float (&ci)[XQ], float (&ch)[XQ]) {
    constexpr int P = C * (C - 1) / 2, QPER = (P + G - 1) / G;
    constexpr int Q0 = GI * QPER < P ? GI * QPER : P;
    constexpr int QN = (Q0 + QPER < P ? Q0 + QPER : P) - Q0;
    float2 u[C];
    float p[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        u[c] = U[c * KB];
        p[c] = u[c].x * u[c].x + u[c].y * u[c].y;
    }
#pragma unroll
    for (int r = 0; r < xs_pmax(G); ++r)
        if constexpr (GI < C) {
            if (GI + G * r < C) pw[r] += p[(GI + G * r) < C ? GI + G * r : 0];
        }
    XsPairs<C, G, GI, COH, 0, QN>::run(u, p, cr, ci, ch);
}

template <int C, int G, bool COH, int GI = 0>
__device__ __forceinline__ void xs_frame_dispatch(int g, const float2* U, int KB, float (&pw)[xs_pmax(G)],
                                                  float (&cr)[XQ], float (&ci)[XQ], float (&ch)[XQ]) {
    if constexpr (GI < G) {
        if (g == GI) xs_frame_static<C, G, GI, COH>(U, KB, pw, cr, ci, ch);
        else xs_frame_dispatch<C, G, COH, GI + 1>(g, U, KB, pw, cr, ci, ch);
    }
}

// CTA (blockIdx.x = bin tile, blockIdx.y = frame slice s) of one chunk of nf
// frames.  part[(s * planes + plane) * nbins + k], planes: C powers, then
// Re and Im of the P cross sums (interleaved per pair), then P per-frame
// coherence sums (only when COH).  first: store, else add.
template <int G, bool COH, int CC = 0>
__global__ void __launch_bounds__(XS_THREADS, 2)
    k_xspec_acc(const float2* __restrict__ X, int C, int nbins, long long nf, int per, int first,
                float* __restrict__ part) {
    // CC > 0: the channel count is the compile-time CC (== C)
    grid_dep_wait();  // the chunk's spectra come from the k_xstft launched just before
    constexpr int KB = XS_THREADS / G, PMAX = xs_pmax(G);
    extern __shared__ __align__(16) float2 stage[];  // [XS_ST][XF][C][KB]
    // byte offsets (channel i, channel j) of every pair inside a frame's
    // [C][KB] block, upper-triangle order (row i holds C - 1 - i pairs)
    __shared__ uint2 pair_off[XS_MAX_PAIRS];
    const int g = threadIdx.x / KB, b = threadIdx.x % KB;
    const int hs = xs_stride(2 * (nbins - 1));
    const int k = blockIdx.x * KB + b;
    const bool live = k < nbins - 1;  // the Nyquist bin n/2 goes through k_xspec_nyq
    const int P = C * (C - 1) / 2;
    const int qper = (P + G - 1) / G;
    const int q0 = min(P, g * qper), qn = min(P, q0 + qper) - q0;
    if (threadIdx.x < P) {
        int r = threadIdx.x, i = 0;
        while (r >= C - 1 - i) r -= C - 1 - i++;
        pair_off[threadIdx.x] = make_uint2(i * KB * 8u, (i + 1 + r) * KB * 8u);
    }
    const int pn = g < C ? (C - g + G - 1) / G : 0;
    float pw[PMAX], cr[XQ], ci[XQ], ch[XQ];
#pragma unroll
    for (int r = 0; r < PMAX; ++r) pw[r] = 0.f;
#pragma unroll
    for (int q = 0; q < XQ; ++q) cr[q] = ci[q] = ch[q] = 0.f;

    const long long fa = (long long)blockIdx.y * per;
    const long long fb = min(nf, fa + per);
    const int nst = fb > fa ? (int)((fb - fa + XF - 1) / XF) : 0;
    const int elems = XF * C * KB;  // float2 per stage
    const int tile0 = blockIdx.x * KB;
    // 16-byte copies of bin pairs (KB, tile0 and nbins - 1 = n/2 are even, so a
    // pair never crosses a row's n/2 + 16 entries)
    auto issue = [&](int si) {
        float2* dst = stage + (si % XS_ST) * elems;
        const long long fs = fa + (long long)si * XF;
        // stage row r = e / KB is frame fs + r / C, channel r % C: global
        // row fs * C + r of the chunk's [frame][channel] spectra
        static_assert((KB & (KB - 1)) == 0, "stage index arithmetic");
        const long long rows_left = (fb - fs) * C;
        const float2* Xs = X + fs * C * hs;
        for (int e = 2 * threadIdx.x; e < elems; e += 2 * XS_THREADS) {
            const int r = e >> ilog2c(KB), bb = e & (KB - 1);
            const bool ok = r < rows_left;
            const int kk = min(tile0 + bb, nbins - 1);
            cp_async16(dst + e, ok ? Xs + (long long)r * hs + kk : X, ok);
        }
    };
    // XS_ST - 1 stages in flight ahead of the one being summed
#pragma unroll
    for (int s0 = 0; s0 < XS_ST - 1; ++s0) {
        if (s0 < nst) issue(s0);
        cp_async_commit_xs();
    }
    __syncthreads();  // pair_off
    for (int si = 0; si < nst; ++si) {
        // refills the buffer summed in the previous iteration (all threads
        // passed its closing barrier)
        if (si + XS_ST - 1 < nst) issue(si + XS_ST - 1);
        cp_async_commit_xs();
        cp_async_wait_xs();
        __syncthreads();
        if (CC > 0 && live) {
#pragma unroll
            for (int fr = 0; fr < XF; ++fr)
                xs_frame_dispatch<(CC > 0 ? CC : 2), G, COH>(g, stage + (si % XS_ST) * elems + fr * CC * KB + b, KB, pw,
                                                            cr, ci, ch);
        } else if (live) {
            const char* U0 = reinterpret_cast<const char*>(stage + (si % XS_ST) * elems + b);
#pragma unroll
            for (int fr = 0; fr < XF; ++fr) {
                const char* U = U0 + fr * C * KB * 8;
#pragma unroll
                for (int r = 0; r < PMAX; ++r)
                    if (r < pn) {
                        const float2 u = *reinterpret_cast<const float2*>(U + (g + G * r) * KB * 8);
                        pw[r] += u.x * u.x + u.y * u.y;
                    }
#pragma unroll
                for (int q = 0; q < XQ; ++q)
                    if (q < qn) {
                        const uint2 o = pair_off[q0 + q];
                        const float2 ui = *reinterpret_cast<const float2*>(U + o.x);
                        const float2 uj = *reinterpret_cast<const float2*>(U + o.y);
                        // S_ij = X_i conj(X_j) (fft_cross_spectral.metal:57-58)
                        const float sr = ui.x * uj.x + ui.y * uj.y;
                        const float sim = ui.y * uj.x - ui.x * uj.y;
                        cr[q] += sr;
                        ci[q] += sim;
                        if constexpr (COH) {
                            const float pi = ui.x * ui.x + ui.y * ui.y, pj = uj.x * uj.x + uj.y * uj.y;
                            ch[q] += (sr * sr + sim * sim) * rcp_approx(fmaxf(pi * pj, 1e-30f));
                        }
                    }
            }
        }
        __syncthreads();
    }
    if (!live) return;
    const int planes = C + (COH ? 3 : 2) * P;
    float* dst = part + (long long)blockIdx.y * planes * nbins + k;  // tiles partition the bins
    auto put = [&](int plane, float v) {
        float* d = dst + (long long)plane * nbins;
        *d = first ? v : *d + v;
    };
#pragma unroll
    for (int r = 0; r < PMAX; ++r)
        if (r < pn) put(g + G * r, pw[r]);
#pragma unroll
    for (int q = 0; q < XQ; ++q)
        if (q < qn) {
            put(C + 2 * (q0 + q), cr[q]);
            put(C + 2 * (q0 + q) + 1, ci[q]);
            if constexpr (COH) put(C + 2 * P + q0 + q, ch[q]);
        }
}

// The Nyquist bin n/2 of every frame of the call (real values nyq[frame][channel]):
// one CTA per item -- items 0 .. C-1 powers sum x_c^2, C .. C+P-1 pair cross
// sums sum x_i x_j, C+P .. C+2P-1 (COH) per-frame coherence sums with the
// pair kernel's FP32 formula.  FP64 sums, each thread over frames t, t+256,
// ..., then a fixed-order tree: deterministic.  Launched with C + P items
// (Welch estimate) or C + 2P (per-frame coherence).
__global__ void __launch_bounds__(256) k_xspec_nyq(const float* __restrict__ nyq, int C, long long frames,
                                                   double* __restrict__ out) {
    const int P = C * (C - 1) / 2, item = blockIdx.x;
    int i = 0, j = 0, kind = 0;  // 0 power, 1 cross, 2 coherence
    if (item < C) {
        i = j = item;
    } else {
        int r = (item - C) % P;
        kind = item < C + P ? 1 : 2;
        while (r >= C - 1 - i) r -= C - 1 - i++;
        j = i + 1 + r;
    }
    double acc = 0.0;
    for (long long f = threadIdx.x; f < frames; f += 256) {
        const float xi = nyq[f * C + i], xj = nyq[f * C + j];
        const float sr = xi * xj;
        if (kind == 2)
            acc += (double)((sr * sr) * rcp_approx(fmaxf((xi * xi) * (xj * xj), 1e-30f)));
        else
            acc += (double)sr;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[item] = red[0];
}

// one thread per (bin k <= n/2, item): items 0 .. C-1 are powers, C .. C+P-1
// pairs.  Fixed-order FP64 sums over the frame slices, / frames, mirrored to n - k.
// COH: coherence = mean of the per-frame values; else the Welch estimate
// |sum S_ij|^2 / (sum p_i sum p_j) (0 where the denominator is not positive).
template <bool COH>
__global__ void k_xspec_finish(const float* __restrict__ part, const double* __restrict__ nyq_sum, int slices, int C,
                               int nbins, long long frames, float* __restrict__ power, float2* __restrict__ cross,
                               float* __restrict__ coh) {
    const int P = C * (C - 1) / 2;
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)(C + P) * nbins) return;
    const int item = (int)(id / nbins), k = (int)(id - (long long)item * nbins);
    const int n = 2 * (nbins - 1);
    const int planes = C + (COH ? 3 : 2) * P;
    const double inv = 1.0 / (double)frames;
    // the Nyquist bin's totals come from k_xspec_nyq: C powers, P cross
    // sums (real), P coherence sums
    const bool nyqk = k == nbins - 1;
    auto sum = [&](int plane) {
        if (nyqk) {
            if (plane < C) return nyq_sum[plane];
            const int r = plane - C;
            if (r < 2 * P) return (r & 1) ? 0.0 : nyq_sum[C + r / 2];
            return nyq_sum[C + P + (r - 2 * P)];
        }
        double s = 0.0;
        for (int u = 0; u < slices; ++u) s += part[((long long)u * planes + plane) * nbins + k];
        return s;
    };
    const int km = (n - k) & (n - 1);
    if (item < C) {
        const float v = (float)(sum(item) * inv);
        power[(long long)item * n + k] = v;
        if (km != k) power[(long long)item * n + km] = v;
        return;
    }
    const int q = item - C;
    const double sr = sum(C + 2 * q), si = sum(C + 2 * q + 1);
    const float2 s = make_float2((float)(sr * inv), (float)(si * inv));
    cross[(long long)q * n + k] = s;
    if (km != k) cross[(long long)q * n + km] = make_float2(s.x, -s.y);
    float c;
    if constexpr (COH) {
        c = (float)(sum(C + 2 * P + q) * inv);
    } else {
        int i = 0, r = q;
        while (r >= C - 1 - i) r -= C - 1 - i++;
        const int j = i + 1 + r;
        const double den = sum(i) * sum(j);
        c = den > 0.0 ? (float)((sr * sr + si * si) / den) : 0.f;
    }
    coh[(long long)q * n + k] = c;
    if (km != k) coh[(long long)q * n + km] = c;
}

struct SpKernels {
    int fft, threads, lines;
    int smem_stft, smem_welch, smem_coh;
    cudaError_t (*prepare)();
    void (*stft)(dim3, cudaStream_t, const float*, long long, int, const float*, const float2*, float2*, float*);
    void (*acc)(bool, dim3, cudaStream_t, const float*, const float*, long long, int, const float*, const float2*,
                long long, long long, float*);
    int (*acc_ctas_per_sm)(bool);
    void (*xstft)(dim3, cudaStream_t, const float*, long long, int, long long, long long, int, const float*,
                  const float2*, float2*, float*);
};

template <int FFT>
cudaError_t sp_prepare() {
    using G = SpGeom<FFT>;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_stft<FFT>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::XCH * 8))) return e;
    if ((e = cudaFuncSetAttribute(k_spec_acc<FFT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  G::template smem_bytes<1>())))
        return e;
    if ((e = cudaFuncSetAttribute(k_xstft<FFT>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::XCH * 8))) return e;
    return cudaFuncSetAttribute(k_spec_acc<FFT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                G::template smem_bytes<4>());
}
template <int FFT>
void sp_xstft(dim3 grid, cudaStream_t s, const float* x, long long len, int C, long long f0, long long nf, int hop,
              const float* w, const float2* tw, float2* X, float* nyq) {
    launch_pdl(k_xstft<FFT>, grid, SpGeom<FFT>::THREADS, SpGeom<FFT>::XCH * 8, s, x, len, C, f0, nf, hop, w, tw, X,
               nyq);
}
template <int FFT>
void sp_stft(dim3 grid, cudaStream_t s, const float* x, long long frames, int hop, const float* w, const float2* tw,
             float2* spec, float* power) {
    k_stft<FFT><<<grid, SpGeom<FFT>::THREADS, SpGeom<FFT>::XCH * 8, s>>>(x, frames, hop, w, tw, spec, power);
}
template <int FFT>
void sp_acc(bool coh, dim3 grid, cudaStream_t s, const float* a, const float* b, long long frames, int hop,
            const float* w, const float2* tw, long long work, long long per, float* part) {
    using G = SpGeom<FFT>;
    if (coh)
        k_spec_acc<FFT, true><<<grid, G::THREADS, G::template smem_bytes<4>(), s>>>(a, b, frames, hop, w, tw, work,
                                                                                    per, part);
    else
        k_spec_acc<FFT, false><<<grid, G::THREADS, G::template smem_bytes<1>(), s>>>(a, b, frames, hop, w, tw, work,
                                                                                     per, part);
}

template <int FFT>
int sp_acc_occ(bool coh) {
    using G = SpGeom<FFT>;
    int occ = 0;
    cudaError_t e = coh ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spec_acc<FFT, true>, G::THREADS,
                                                                        G::template smem_bytes<4>())
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spec_acc<FFT, false>, G::THREADS,
                                                                        G::template smem_bytes<1>());
    return (e == cudaSuccess && occ > 0) ? occ : 1;
}

#define MFFT_SPK(F)                                                                                         \
    {F, SpGeom<F>::THREADS, SpGeom<F>::LINES, SpGeom<F>::XCH * 8, SpGeom<F>::template smem_bytes<1>(),     \
     SpGeom<F>::template smem_bytes<4>(), &sp_prepare<F>, &sp_stft<F>, &sp_acc<F>, &sp_acc_occ<F>, &sp_xstft<F>}

const SpKernels g_spk[] = {MFFT_SPK(64),   MFFT_SPK(128),  MFFT_SPK(256),  MFFT_SPK(512),  MFFT_SPK(1024),
                           MFFT_SPK(2048), MFFT_SPK(4096), MFFT_SPK(8192), MFFT_SPK(16384)};

const SpKernels* find_spk(int fft) {
    for (const auto& k : g_spk)
        if (k.fft == fft) return &k;
    return nullptr;
}

template <int G, bool COH, int CC = 0>
void xs_launch(dim3 grid, int smem, cudaStream_t s, const float2* X, int C, int nbins, long long nf, int per,
               int first, float* part) {
    launch_pdl(k_xspec_acc<G, COH, CC>, grid, XS_THREADS, smem, s, X, C, nbins, nf, per, first, part);
}
using XsFn = void (*)(dim3, int, cudaStream_t, const float2*, int, int, long long, int, int, float*);
// channel counts 2, 4 and 8 have a compile-time kernel (G = xs_groups(C))
XsFn xs_fn(int g, bool coh, int C) {
    switch (C) {  // g == xs_groups(C): 1, 1, 4
        case 2: return coh ? &xs_launch<1, true, 2> : &xs_launch<1, false, 2>;
        case 4: return coh ? &xs_launch<1, true, 4> : &xs_launch<1, false, 4>;
        case 8: return coh ? &xs_launch<4, true, 8> : &xs_launch<4, false, 8>;
        default: break;
    }
    switch (g) {
        case 1: return coh ? &xs_launch<1, true> : &xs_launch<1, false>;
        case 2: return coh ? &xs_launch<2, true> : &xs_launch<2, false>;
        case 4: return coh ? &xs_launch<4, true> : &xs_launch<4, false>;
        case 8: return coh ? &xs_launch<8, true> : &xs_launch<8, false>;
        default: return coh ? &xs_launch<16, true> : &xs_launch<16, false>;
    }
}
// shared-memory opt-in on the current device, then the resident CTAs per SM
// (0 when the opt-in fails)
template <int G, bool COH, int CC = 0>
int xs_occ_of(int smem) {
    if (cudaFuncSetAttribute(k_xspec_acc<G, COH, CC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
        return 0;
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_xspec_acc<G, COH, CC>, XS_THREADS, smem);
    return (e == cudaSuccess && occ > 0) ? occ : 1;
}
int xs_occ(int g, bool coh, int smem, int C) {
    switch (C) {
        case 2: return coh ? xs_occ_of<1, true, 2>(smem) : xs_occ_of<1, false, 2>(smem);
        case 4: return coh ? xs_occ_of<1, true, 4>(smem) : xs_occ_of<1, false, 4>(smem);
        case 8: return coh ? xs_occ_of<4, true, 8>(smem) : xs_occ_of<4, false, 8>(smem);
        default: break;
    }
    switch (g) {
        case 1: return coh ? xs_occ_of<1, true>(smem) : xs_occ_of<1, false>(smem);
        case 2: return coh ? xs_occ_of<2, true>(smem) : xs_occ_of<2, false>(smem);
        case 4: return coh ? xs_occ_of<4, true>(smem) : xs_occ_of<4, false>(smem);
        case 8: return coh ? xs_occ_of<8, true>(smem) : xs_occ_of<8, false>(smem);
        default: return coh ? xs_occ_of<16, true>(smem) : xs_occ_of<16, false>(smem);
    }
}

// spectra of one chunk stay at most this large (L2 holds them until the
// accumulation reads them back; 8 channels at fftSize 1024: 48 MiB chunks
// 0.636 ms per call, 32 MiB 0.675 ms, 64 MiB 0.649 ms)
constexpr long long XS_CHUNK_BYTES = 48ll << 20;

}  // namespace

}  // namespace mfft

using namespace mfft;

struct mfft_spectral {
    mfft_ctx* ctx = nullptr;
    int64_t fft = 0, hop = 0;
    const SpKernels* k = nullptr;
    float2* tw = nullptr;
    float* window = nullptr;  // device
    double window_sumsq = 0;
    float* part = nullptr;    // walker sums
    long long part_floats = 0;
    int occ_welch = 0, occ_coh = 0;  // resident CTAs per SM of the accumulation kernels
    float2* xs_spec = nullptr;        // cross-spectral: spectra of one chunk
    long long xs_spec_elems = 0;
    float* xs_part = nullptr;         // cross-spectral: sums per frame slice
    long long xs_part_floats = 0;
    float* xs_nyq = nullptr;          // cross-spectral: Nyquist bin of every frame and channel
    long long xs_nyq_floats = 0;
    double* xs_nyq_sum = nullptr;     // cross-spectral: the Nyquist bin's totals
    long long xs_nyq_sums = 0;
};

extern "C" int mfft_spectral_destroy(mfft_spectral* s) {
    if (!s) return MFFT_SUCCESS;
    DeviceGuard g(s->ctx->device);
    cudaFree(s->window);
    cudaFree(s->part);
    cudaFree(s->xs_spec);
    cudaFree(s->xs_part);
    cudaFree(s->xs_nyq);
    cudaFree(s->xs_nyq_sum);
    delete s;
    return MFFT_SUCCESS;
}

extern "C" int mfft_spectral_create(mfft_ctx* ctx, int64_t fft_size, int64_t hop_size, int window_kind,
                                    double kaiser_beta, mfft_spectral** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    *out = nullptr;
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    if (!is_pow2_in(fft_size, 64, MFFT_MAX_SINGLE_N))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, fft_size, -1, -1,
                         "Unsupported FFT size: %lld. Supported: powers of two 64..16384", (long long)fft_size);
    if (hop_size < 1 || hop_size > (1LL << 30))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, hop_size, -1, "hop size must be in [1, 2^30], got %lld",
                         (long long)hop_size);
    std::vector<float> w((size_t)fft_size);
    int st = mfft_window(window_kind, fft_size, kaiser_beta, w.data());
    if (st) return st;
    DeviceGuard g(ctx->device);
    mfft_spectral* s = new mfft_spectral();
    s->ctx = ctx;
    s->fft = fft_size;
    s->hop = hop_size;
    s->k = find_spk((int)fft_size);
    for (float v : w) s->window_sumsq += (double)v * (double)v;
    st = line_twiddles(ctx, (int)fft_size, &s->tw);
    cudaError_t e = cudaSuccess;
    if (!st) e = s->k->prepare();
    if (!st && e != cudaSuccess) st = cuda_error(e, "spectral kernel attributes");
    if (!st) {
        e = cudaMalloc(&s->window, sizeof(float) * fft_size);
        if (e == cudaSuccess) e = cudaMemcpy(s->window, w.data(), sizeof(float) * fft_size, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "window: %s", cudaGetErrorString(e));
    }
    if (st) {
        mfft_spectral_destroy(s);
        return st;
    }
    *out = s;
    return MFFT_SUCCESS;
}

extern "C" int64_t mfft_stft_frame_count(const mfft_spectral* s, int64_t sample_count) {
    if (!s || sample_count < s->fft) return 0;
    return (sample_count - s->fft) / s->hop + 1;
}

namespace {

// Host-array call with several inputs and outputs: stage, run, copy back, wait.
struct HostBuf {
    const void* host_in;
    void* host_out;
    size_t bytes;
    void* dev;
};
int host_call(mfft_ctx* ctx, std::vector<HostBuf>& bufs, const std::function<int(cudaStream_t)>& body) {
    cudaStream_t s = ctx->stream;
    int st = MFFT_SUCCESS;
    cudaError_t e = cudaSuccess;
    for (auto& b : bufs) {
        b.dev = nullptr;
        if (!b.bytes) continue;
        e = cudaMallocAsync(&b.dev, b.bytes, s);
        if (e != cudaSuccess) {
            st = set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "Device buffer allocation failed: %s", cudaGetErrorString(e));
            break;
        }
        if (b.host_in) {
            e = cudaMemcpyAsync(b.dev, b.host_in, b.bytes, cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) {
                st = cuda_error(e, "host to device copy");
                break;
            }
        }
    }
    if (!st) st = body(s);
    if (!st)
        for (auto& b : bufs)
            if (b.host_out && b.dev) {
                e = cudaMemcpyAsync(b.host_out, b.dev, b.bytes, cudaMemcpyDeviceToHost, s);
                if (e != cudaSuccess) {
                    st = cuda_error(e, "device to host copy");
                    break;
                }
            }
    for (auto& b : bufs)
        if (b.dev) cudaFreeAsync(b.dev, s);
    e = cudaStreamSynchronize(s);
    if (!st && e != cudaSuccess) st = cuda_error(e, "execution");
    if (!st) st = check_device_error(ctx);
    return st;
}

int check_flags(int flags) {
    if (flags != MFFT_HOST_MEMORY && flags != MFFT_DEVICE_MEMORY)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown flags %d", flags);
    return MFFT_SUCCESS;
}

int stft_device(mfft_spectral* s, const float* x, long long frames, float2* spec, float* power, cudaStream_t st) {
    const long long pairs = (frames + 1) / 2;
    const long long ctas = (pairs + s->k->lines - 1) / s->k->lines;
    if (ctas <= 0) return MFFT_SUCCESS;
    if (ctas > 0x7fffffffLL) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, frames, -1, "too many frames");
    s->k->stft(dim3((unsigned)ctas), st, x, frames, (int)s->hop, s->window, s->tw, spec, power);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "STFT launch");
    return MFFT_SUCCESS;
}

// walkers over `work` items (pairs or frames): one CTA per resident slot
int acc_device(mfft_spectral* s, bool coh, const float* a, const float* b, long long frames, long long work,
               float scale, float* out, cudaStream_t st) {
    const int lines = s->k->lines;
    int& occ = coh ? s->occ_coh : s->occ_welch;
    if (!occ) occ = s->k->acc_ctas_per_sm(coh);
    long long units = (long long)s->ctx->sms * occ * lines;
    if (units > work) units = work;
    if (units < 1) units = 1;
    const long long per = work > 0 ? (work + units - 1) / units : 0;
    units = per > 0 ? (work + per - 1) / per : 1;
    const long long ctas = (units + lines - 1) / lines;
    const long long slots = ctas * lines;
    const int planes = coh ? 4 : 1;
    const long long need = slots * planes * s->fft;
    if (need > s->part_floats) {
        cudaFree(s->part);
        s->part = nullptr;
        s->part_floats = 0;
        cudaError_t e = cudaMalloc(&s->part, sizeof(float) * need);
        if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "spectral sums: %s", cudaGetErrorString(e));
        s->part_floats = need;
    }
    s->k->acc(coh, dim3((unsigned)ctas), st, a, b, frames, (int)s->hop, s->window, s->tw, work, per, s->part);
    const unsigned fin = (unsigned)(s->fft / FIN_BINS);
    if (coh) k_spec_finish<true><<<fin, FIN_BINS * FIN_RUNS, 0, st>>>(s->part, slots, (int)s->fft, scale, out);
    else k_spec_finish<false><<<fin, FIN_BINS * FIN_RUNS, 0, st>>>(s->part, slots, (int)s->fft, scale, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "spectral launch");
    return MFFT_SUCCESS;
}

}  // namespace

extern "C" int mfft_stft_analyze(mfft_spectral* s, const float* signal, int64_t n, void* spectra, float* power,
                                 int flags, void* stream) {
    if (!s) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "spectral handle is NULL");
    int st = check_flags(flags);
    if (st) return st;
    if (n < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, n, -1, "signal length must be >= 0");
    const long long frames = mfft_stft_frame_count(s, n);
    if (frames > 0 && !signal) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL signal");
    if (frames == 0) return MFFT_SUCCESS;
    DeviceGuard g(s->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY)
        return stft_device(s, signal, frames, (float2*)spectra, power, (cudaStream_t)stream);
    const size_t nb = (size_t)frames * s->fft;
    std::vector<HostBuf> bufs = {{signal, nullptr, (size_t)n * 4, nullptr},
                                 {nullptr, spectra, spectra ? nb * 8 : 0, nullptr},
                                 {nullptr, power, power ? nb * 4 : 0, nullptr}};
    return host_call(s->ctx, bufs, [&](cudaStream_t cs) {
        return stft_device(s, (const float*)bufs[0].dev, frames, (float2*)bufs[1].dev, (float*)bufs[2].dev, cs);
    });
}

extern "C" int mfft_psd_welch(mfft_spectral* s, const float* signal, int64_t n, double sample_rate, float* psd,
                              int flags, void* stream) {
    if (!s) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "spectral handle is NULL");
    int st = check_flags(flags);
    if (st) return st;
    if (n < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, n, -1, "signal length must be >= 0");
    if (!psd) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL output");
    const long long frames = mfft_stft_frame_count(s, n);
    if (frames > 0 && !signal) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL signal");
    // PSD.swift:53-56: 1 / (frames * sum(w^2) * sampleRate); no frames: zeros
    const float scale = frames > 0 ? (float)(1.0 / ((double)frames * s->window_sumsq * sample_rate)) : 0.f;
    DeviceGuard g(s->ctx->device);
    const long long pairs = (frames + 1) / 2;
    if (flags == MFFT_DEVICE_MEMORY) {
        if (frames == 0) {
            cudaError_t e = cudaMemsetAsync(psd, 0, sizeof(float) * s->fft, (cudaStream_t)stream);
            return e == cudaSuccess ? MFFT_SUCCESS : cuda_error(e, "PSD zero fill");
        }
        return acc_device(s, false, signal, nullptr, frames, pairs, scale, psd, (cudaStream_t)stream);
    }
    std::vector<HostBuf> bufs = {{signal, nullptr, frames > 0 ? (size_t)n * 4 : 0, nullptr},
                                 {nullptr, psd, (size_t)s->fft * 4, nullptr}};
    return host_call(s->ctx, bufs, [&](cudaStream_t cs) {
        if (frames == 0) {
            cudaError_t e = cudaMemsetAsync(bufs[1].dev, 0, sizeof(float) * s->fft, cs);
            return e == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(e, "PSD zero fill");
        }
        return acc_device(s, false, (const float*)bufs[0].dev, nullptr, frames, pairs, scale, (float*)bufs[1].dev, cs);
    });
}

extern "C" int mfft_psd_coherence(mfft_spectral* s, const float* a, int64_t na, const float* b, int64_t nb,
                                  float* coherence, int flags, void* stream) {
    if (!s) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "spectral handle is NULL");
    int st = check_flags(flags);
    if (st) return st;
    if (na < 0 || nb < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "signal lengths must be >= 0");
    if (!coherence) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL output");
    const long long n = na < nb ? na : nb;  // PSD.swift:98
    const long long frames = mfft_stft_frame_count(s, n);
    if (frames > 0 && (!a || !b)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL signal");
    DeviceGuard g(s->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY) {
        if (frames == 0) {
            cudaError_t e = cudaMemsetAsync(coherence, 0, sizeof(float) * s->fft, (cudaStream_t)stream);
            return e == cudaSuccess ? MFFT_SUCCESS : cuda_error(e, "coherence zero fill");
        }
        return acc_device(s, true, a, b, frames, frames, 1.f, coherence, (cudaStream_t)stream);
    }
    const size_t in_b = frames > 0 ? (size_t)n * 4 : 0;
    std::vector<HostBuf> bufs = {{a, nullptr, in_b, nullptr},
                                 {b, nullptr, in_b, nullptr},
                                 {nullptr, coherence, (size_t)s->fft * 4, nullptr}};
    return host_call(s->ctx, bufs, [&](cudaStream_t cs) {
        if (frames == 0) {
            cudaError_t e = cudaMemsetAsync(bufs[2].dev, 0, sizeof(float) * s->fft, cs);
            return e == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(e, "coherence zero fill");
        }
        return acc_device(s, true, (const float*)bufs[0].dev, (const float*)bufs[1].dev, frames, frames, 1.f,
                          (float*)bufs[2].dev, cs);
    });
}

namespace {

int grow(void** p, long long& have, long long need, size_t elem, const char* what) {
    if (need <= have) return MFFT_SUCCESS;
    cudaFree(*p);
    *p = nullptr;
    have = 0;
    cudaError_t e = cudaMalloc(p, elem * (size_t)need);
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "%s: %s", what, cudaGetErrorString(e));
    have = need;
    return MFFT_SUCCESS;
}

int xspec_device(mfft_spectral* s, const float* x, int C, long long len, float* power, float2* cross, float* coh,
                 int mode, cudaStream_t st) {
    const int fft = (int)s->fft, nbins = fft / 2 + 1, hs = xs_stride(fft);
    const int P = C * (C - 1) / 2;
    const long long frames = mfft_stft_frame_count(s, len);
    cudaError_t e;
    if (frames == 0) {  // CrossSpectral.swift:130-133: zero accumulators
        e = cudaMemsetAsync(power, 0, sizeof(float) * C * fft, st);
        if (e == cudaSuccess && P) e = cudaMemsetAsync(cross, 0, sizeof(float2) * P * fft, st);
        if (e == cudaSuccess && P) e = cudaMemsetAsync(coh, 0, sizeof(float) * P * fft, st);
        return e == cudaSuccess ? MFFT_SUCCESS : cuda_error(e, "cross-spectral zero fill");
    }
    const bool per_frame = mode == 0;
    const int g = xs_groups(C), kb = XS_THREADS / g, smem = xs_smem(C, g);
    if ((C + g - 1) / g > xs_pmax(g) || (P + g - 1) / g > XQ)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, C, -1, "channel split %d does not fit", g);
    const int tiles = (nbins - 1 + kb - 1) / kb;  // bins 0 .. n/2 - 1; n/2 by k_xspec_nyq
    // frames per chunk: even, at most XS_CHUNK_BYTES of spectra, no more than needed
    long long fch = XS_CHUNK_BYTES / ((long long)C * hs * 8);
    fch = fch < 2 ? 2 : fch & ~1LL;
    if (fch > frames + (frames & 1)) fch = frames + (frames & 1);
    // frame slices: enough CTAs to fill the GPU once over the bin tiles
    const int occ = xs_occ(g, per_frame, smem, C);
    if (!occ) return cuda_error(cudaGetLastError(), "cross-spectral kernel attributes");
    long long slices = ((long long)s->ctx->sms * occ + tiles - 1) / tiles;
    const long long max_slices = (fch + XF - 1) / XF;
    if (slices > max_slices) slices = max_slices;
    if (slices < 1) slices = 1;
    long long per = (fch + slices - 1) / slices;
    per = (per + XF - 1) / XF * XF;
    slices = (fch + per - 1) / per;
    const int planes = C + (per_frame ? 3 : 2) * P;
    int rc = grow((void**)&s->xs_spec, s->xs_spec_elems, fch * C * hs, sizeof(float2), "cross-spectral spectra");
    if (!rc) rc = grow((void**)&s->xs_part, s->xs_part_floats, slices * planes * nbins, sizeof(float),
                       "cross-spectral sums");
    if (!rc) rc = grow((void**)&s->xs_nyq, s->xs_nyq_floats, (frames + 1) * C, sizeof(float),
                       "cross-spectral Nyquist bins");
    if (!rc) rc = grow((void**)&s->xs_nyq_sum, s->xs_nyq_sums, C + 2 * P, sizeof(double),
                       "cross-spectral Nyquist sums");
    if (rc) return rc;
    const XsFn acc = xs_fn(g, per_frame, C);
    for (long long f0 = 0; f0 < frames; f0 += fch) {
        const long long nf = frames - f0 < fch ? frames - f0 : fch;
        const long long lines = (long long)C * ((nf + 1) / 2);
        const long long ctas = (lines + s->k->lines - 1) / s->k->lines;
        s->k->xstft(dim3((unsigned)ctas), st, x, len, C, f0, nf, (int)s->hop, s->window, s->tw, s->xs_spec,
                    s->xs_nyq);
        acc(dim3((unsigned)tiles, (unsigned)slices), smem, st, s->xs_spec, C, nbins, nf, (int)per, f0 == 0,
            s->xs_part);
    }
    k_xspec_nyq<<<(unsigned)(C + (per_frame ? 2 : 1) * P), 256, 0, st>>>(s->xs_nyq, C, frames, s->xs_nyq_sum);
    const long long items = (long long)(C + P) * nbins;
    if (per_frame)
        k_xspec_finish<true><<<(unsigned)((items + 255) / 256), 256, 0, st>>>(
            s->xs_part, s->xs_nyq_sum, (int)slices, C, nbins, frames, power, cross, coh);
    else
        k_xspec_finish<false><<<(unsigned)((items + 255) / 256), 256, 0, st>>>(
            s->xs_part, s->xs_nyq_sum, (int)slices, C, nbins, frames, power, cross, coh);
    e = cudaGetLastError();
    return e == cudaSuccess ? MFFT_SUCCESS : cuda_error(e, "cross-spectral launch");
}

}  // namespace

extern "C" int mfft_psd_cross_spectral(mfft_spectral* s, const float* signals, int64_t channels, int64_t length,
                                       float* power, void* cross, float* coherence, int coherence_mode, int flags,
                                       void* stream) {
    if (!s) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "spectral handle is NULL");
    int st = check_flags(flags);
    if (st) return st;
    // CrossSpectral.swift:63-66: 1..16 channels of one length
    if (channels < 1 || channels > XS_MAX_CH)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, channels, -1, "crossSpectral requires 1-16 channels, got %lld",
                         (long long)channels);
    if (length < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, length, -1, "signal length must be >= 0");
    if (coherence_mode != 0 && coherence_mode != 1)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, coherence_mode, -1, "unknown coherence mode %d", coherence_mode);
    const int C = (int)channels, P = C * (C - 1) / 2;
    if (!power || (P && (!cross || !coherence)))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL output");
    const long long frames = mfft_stft_frame_count(s, length);
    if (frames > 0 && !signals) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL signal");
    if (frames > 0 && (long long)C * length > (1LL << 40))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, length, -1, "signals too long");
    DeviceGuard g(s->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY)
        return xspec_device(s, signals, C, length, power, (float2*)cross, coherence, coherence_mode,
                            (cudaStream_t)stream);
    const size_t fft = (size_t)s->fft;
    std::vector<HostBuf> bufs = {{signals, nullptr, frames > 0 ? (size_t)C * length * 4 : 0, nullptr},
                                 {nullptr, power, (size_t)C * fft * 4, nullptr},
                                 {nullptr, cross, (size_t)P * fft * 8, nullptr},
                                 {nullptr, coherence, (size_t)P * fft * 4, nullptr}};
    return host_call(s->ctx, bufs, [&](cudaStream_t cs) {
        return xspec_device(s, (const float*)bufs[0].dev, C, length, (float*)bufs[1].dev, (float2*)bufs[2].dev,
                            (float*)bufs[3].dev, coherence_mode, cs);
    });
}
