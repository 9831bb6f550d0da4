// conv.cu -- fused overlap-add FIR convolution (Convolver / FusedConvolver)
// and its adjoint, plus the Correlator and FFTAnalyzer line kernels.
//
// Reference: Convolver.apply (Sources/MetalFFT/DSP/Convolve.swift:36-76) runs,
// per block of hop = fft - K + 1 samples, one GPU forward FFT, a CPU complex
// multiply by the kernel spectrum, one GPU inverse FFT and a CPU overlap-add
// of the real parts; FusedConvolver (FusedConvolver.swift:91-133,
// Resources/fft_fused_convolve.metal:113-146) fuses FFT * H * IFFT into one
// dispatch per block (fft = 4096 only).  Here one launch covers the whole
// signal:
//
//  forward   blocks b and b+1 travel as the real and imaginary parts of one
//            complex line (h is real, so IFFT(FFT(x_b + i x_{b+1}) H) =
//            (x_b (*) h) + i (x_{b+1} (*) h)): half the transforms of the
//            reference.  A CTA walks a contiguous range of block pairs and
//            carries the overlap (fft - hop samples) in shared memory; it
//            first recomputes the few blocks before its range that still
//            overlap it.  Every output sample is written once, in order of
//            blocks: no atomics, no zero fill, deterministic.
//  backward  for L with g = dL/dy: dx[n] = sum_k g[n+k] h[k] and
//            dh[k] = sum_n g[n+k] x[n].  Per x block b, one complex line
//            z = g[b*hop, b*hop + fft) + i x_b is transformed; its Hermitian
//            parts give G and X.  dx over the block is IFFT(G conj(H))[0, hop)
//            (a correlation window needs no overlap-add); the dh spectrum
//            sum_b G conj(X) accumulates in registers (each thread owns fixed
//            bins across blocks) and is written per CTA, then summed in a
//            fixed order and inverse-transformed once.  Spectra are
//            recomputed from x and g, never stored per block.
#include <vector>

#include "capi_internal.h"
#include "stockham.cuh"

namespace mfft {

namespace {

constexpr int CONV_E = 16;

template <int FFT>
struct ConvGeom {
    static constexpr int T = FFT / CONV_E;
    static constexpr int LINES = T >= 128 ? 1 : 128 / T;  // independent walkers per CTA
    static constexpr int THREADS = T * LINES;
    static constexpr bool WS = (T <= 32);
    // per line: exchange area (padded) + two overlap accumulators (forward) or
    // the dh spectrum accumulator (backward): FFT x 8 bytes either way.  When
    // that does not fit next to the exchange area (FFT = 16384) the
    // accumulators live in a per-walker global scratch (L2-resident).
    static constexpr int SMEM_F2 = LINES * spad_size(FFT);
    static constexpr bool ACC_SMEM = SMEM_F2 * 8 + LINES * 2 * FFT * 4 <= 227 * 1024;
    static constexpr int SMEM_BYTES = SMEM_F2 * 8 + (ACC_SMEM ? LINES * 2 * FFT * 4 : 0);
    // backward: block 0's dx spectrum waits in shared memory (not in
    // registers) while block 1 is transformed, where it fits
    static constexpr bool STASH = ACC_SMEM && SMEM_BYTES + LINES * FFT * 8 <= 227 * 1024;
    static constexpr int SMEM_BYTES_BWD = SMEM_BYTES + (STASH ? LINES * FFT * 8 : 0);
    // forward CTAs of <= 256 threads run two per SM at 128 registers a
    // thread; the backward kernel needs more registers than that and keeps
    // one CTA per SM (measured: fft 4096 forward 15 % faster at two, backward
    // 24 % slower)
    static constexpr int MINB_FWD = THREADS <= 256 ? 2 : 1;
};

// number of valid samples in a window of `cap` when `avail` remain (0 .. cap)
__device__ __forceinline__ int clamp_count(long long avail, int cap) {
    return avail <= 0 ? 0 : (avail >= cap ? cap : (int)avail);
}

template <bool WS>
__device__ __forceinline__ void cta_sync() {
    __syncthreads();
}

// forward: y[0, ny) from x[0, nx); H = FFT(h zero-padded), natural order.
// Unit u (a walker) owns block pairs [p0, p1) of nout blocks (virtual blocks
// past nx read zeros, so the last overlap is flushed by the same code).
template <int FFT>
__global__ void __launch_bounds__(ConvGeom<FFT>::THREADS, ConvGeom<FFT>::MINB_FWD)
    k_conv_fwd(const float* __restrict__ x, long long nx, float* __restrict__ y, long long ny,
               const float2* __restrict__ H, const float2* __restrict__ tw, int hop, long long npairs,
               long long pairs_per_unit, int warm_blocks, float* __restrict__ acc_g) {
    using G = ConvGeom<FFT>;
    constexpr int T = G::T;
    extern __shared__ __align__(16) float2 smem[];
    const int lf = threadIdx.x / T;
    const int t = threadIdx.x % T;
    const PadLine buf{smem + lf * spad_size(FFT)};
    const long long unit = (long long)blockIdx.x * G::LINES + lf;
    float* acc0 = G::ACC_SMEM ? reinterpret_cast<float*>(smem + G::SMEM_F2) + lf * 2 * FFT : acc_g + unit * 2 * FFT;
    float* acc1 = acc0 + FFT;

    const long long p0 = unit * pairs_per_unit;
    long long p1 = p0 + pairs_per_unit;
    if (p1 > npairs) p1 = npairs;
    long long pw = (2 * p0 - warm_blocks) / 2;
    if (pw < 0) pw = 0;
    if (p0 >= npairs) pw = p1 = 0;  // idle walker (still joins the barriers)

    for (int i = t; i < FFT; i += T) {
        acc0[i] = 0.f;
        acc1[i] = 0.f;
    }
    // all walkers of the CTA iterate the same number of times
    const long long iters_mine = p1 - pw;
    const long long iters = pairs_per_unit + (warm_blocks + 1) / 2 + 1;
    const float sc = 1.0f / (float)FFT;
    __syncthreads();

    for (long long it = 0; it < iters; ++it) {
        const bool active = it < iters_mine;
        const long long p = pw + it;
        const long long b = 2 * p;
        // 32-bit offsets from the pair's base: lim0 / lim1 = valid samples of blocks b, b+1
        const long long base = b * hop;
        const float* xb = x + base;
        const int lim0 = active ? clamp_count(nx - base, hop) : 0;
        const int lim1 = active ? clamp_count(nx - base - hop, hop) : 0;
        float2 v[CONV_E];
#pragma unroll
        for (int m = 0; m < CONV_E; ++m) {
            const int i = t + m * T;
            float re = 0.f, im = 0.f;
            if (i < lim0) re = __ldcs(xb + i);
            if (i < lim1) im = __ldcs(xb + hop + i);
            v[m] = make_float2(re, im);
        }
        // forward transform, times H, inverse transform through one call site
        // (two inlined transforms get interleaved and need more registers)
#pragma unroll 1
        for (int ph = 0; ph < 2; ++ph) {
            fft_regs<FFT, CONV_E, G::WS>(v, t, buf, tw);
            if (ph == 0) {
#pragma unroll
                for (int m = 0; m < CONV_E; ++m) {
                    const float2 h = __ldg(H + t + m * T);
                    v[m] = cconj(cmul(v[m], h));  // conj for the inverse
                }
            }
        }
        // v[m] = conj(FFT * FFT) -> r = conj(v)/FFT; re = block b, im = block b+1
        const bool write = active && p >= p0;
        float* yb = y + base;
        const int wlim0 = write ? clamp_count(ny - base, hop) : 0;
        const int wlim1 = write ? clamp_count(ny - base - hop, hop) : 0;
#pragma unroll
        for (int m = 0; m < CONV_E; ++m) {
            const int i = t + m * T;
            const float val = v[m].x * sc + acc0[i];
            if (i < hop) {
                if (i < wlim0) __stcs(yb + i, val);
            } else {
                acc1[i - hop] = val;
            }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < CONV_E; ++m) {
            const int i = t + m * T;
            const float val = -v[m].y * sc + acc1[i];
            if (i < hop) {
                if (i < wlim1) __stcs(yb + hop + i, val);
            } else {
                acc0[i - hop] = val;
            }
        }
        __syncthreads();
    }
}

// backward: dx[0, nx) and per-walker partial dh spectra part[unit][FFT].
// Blocks b, b+1 travel together, like the forward kernel's pairs:
//   Z = FFT(g_b + i g_{b+1})   (windows of FFT samples of g from b*hop)
//   W = FFT(x_b + i x_{b+1})   (hop samples of x each, zero-padded)
//   dx_b + i dx_{b+1} = IFFT(Z conj H) on [0, hop)   (h real: both halves real)
//   P += Z conj(W)
// With G_b, X_b the Hermitian parts of Z and W, G_b conj X_b + G_{b+1} conj
// X_{b+1} = (P_k + conj P_{-k}) / 2, so the symmetrisation is done once, on
// the summed spectrum (k_dh_finish), and no block needs a Hermitian split.
// Z waits in shared memory (or in this walker's global stash row `zs` when
// shared memory is full) while W is transformed: one 16-value array is live
// at a time.  dx == nullptr skips the dx transform.
template <int FFT>
__global__ void __launch_bounds__(ConvGeom<FFT>::THREADS, 1)
    k_conv_bwd(const float* __restrict__ x, long long nx, const float* __restrict__ g, long long ny,
               const float2* __restrict__ H, const float2* __restrict__ tw, int hop, long long nblocks,
               long long blocks_per_unit, float* __restrict__ dx, float2* __restrict__ part,
               float2* __restrict__ zs) {
    // the dh spectrum accumulates in shared memory, or directly in this
    // walker's row of `part` when shared memory is too small
    using G = ConvGeom<FFT>;
    constexpr int T = G::T;
    extern __shared__ __align__(16) float2 smem[];
    const int lf = threadIdx.x / T;
    const int t = threadIdx.x % T;
    const PadLine buf{smem + lf * spad_size(FFT)};
    const long long unit = (long long)blockIdx.x * G::LINES + lf;
    const long long b0 = unit * blocks_per_unit;
    long long b1 = b0 + blocks_per_unit;
    if (b1 > nblocks) b1 = nblocks;
    const long long mine = b1 > b0 ? b1 - b0 : 0;
    const float sc = 1.0f / (float)FFT;

    // P accumulator and Z stash: bin k at D[k] / Zs[k], owned by one thread
    float2* D = G::ACC_SMEM ? smem + G::SMEM_F2 + lf * FFT : part + unit * FFT;
    float2* Zs = G::STASH ? smem + G::SMEM_F2 + G::LINES * FFT + lf * FFT : zs + unit * FFT;
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) D[t + m * T] = make_float2(0.f, 0.f);

    // this walker's span from one base pointer each, 32-bit offsets inside it
    const long long ubase = b0 * hop;
    const float* gu = g + ubase;
    const float* xu = x + ubase;
    float* du = dx ? dx + ubase : nullptr;
    const long long ny_u = ny - ubase, nx_u = nx - ubase;
    for (int it = 0; it < blocks_per_unit; it += 2) {
        const int off0 = it * hop, off1 = off0 + hop;
        const bool a0 = it < mine, a1 = it + 1 < mine;
        const int ly0 = a0 ? clamp_count(ny_u - off0, FFT) : 0, ly1 = a1 ? clamp_count(ny_u - off1, FFT) : 0;
        const int lx0 = a0 ? clamp_count(nx_u - off0, hop) : 0, lx1 = a1 ? clamp_count(nx_u - off1, hop) : 0;
        // The three transforms of a block pair go through one call site (phase
        // 0: Z, 1: dx, 2: W), so that the compiler does not interleave their
        // code, which needs more registers than a thread of 512 has.
#pragma unroll 1
        for (int ph = 0; ph < 3; ++ph) {
            if (ph == 1 && !du) continue;  // the same for every thread
            float2 v[CONV_E];
            if (ph == 0) {
#pragma unroll
                for (int m = 0; m < CONV_E; ++m) {
                    const int i = t + m * T;
                    v[m] = make_float2(i < ly0 ? __ldcs(gu + off0 + i) : 0.f, i < ly1 ? __ldcs(gu + off1 + i) : 0.f);
                }
            } else if (ph == 1) {
                // conj(Z conj H): the inverse as a forward transform of the conjugate
#pragma unroll
                for (int m = 0; m < CONV_E; ++m) {
                    const int k = t + m * T;
                    v[m] = cconj(cmul(Zs[k], cconj(__ldg(H + k))));
                }
            } else {
#pragma unroll
                for (int m = 0; m < CONV_E; ++m) {
                    const int i = t + m * T;
                    v[m] = make_float2(i < lx0 ? __ldcs(xu + off0 + i) : 0.f, i < lx1 ? __ldcs(xu + off1 + i) : 0.f);
                }
            }
            fft_regs<FFT, CONV_E, G::WS>(v, t, buf, tw);
            if (ph == 0) {
#pragma unroll
                for (int m = 0; m < CONV_E; ++m) Zs[t + m * T] = v[m];
            } else if (ph == 1) {
#pragma unroll
                for (int m = 0; m < CONV_E; ++m) {
                    const int i = t + m * T;
                    // IFFT = conj(FFT(conj)) / FFT: re = block b, im = block b+1
                    if (i < lx0) __stcs(du + off0 + i, v[m].x * sc);
                    if (i < lx1) __stcs(du + off1 + i, -v[m].y * sc);
                }
            } else {
                // P += Z conj(W) (each thread owns its bins)
#pragma unroll
                for (int m = 0; m < CONV_E; ++m) {
                    const int k = t + m * T;
                    D[k] = cadd(D[k], cmul(Zs[k], cconj(v[m])));
                }
            }
        }
    }
    if constexpr (G::ACC_SMEM) {
        float2* dst = part + unit * FFT;
#pragma unroll
        for (int m = 0; m < CONV_E; ++m) dst[t + m * T] = D[t + m * T];
    }
}

// sum of the walkers' dh spectra in a fixed order: a CTA owns 16 consecutive
// bins; thread (run r, bin b) sums walkers [r*R, (r+1)*R) of its bin in walker
// order, then lane b adds the 16 runs in run order (fft/16 CTAs)
constexpr int SUM_BINS = 16, SUM_RUNS = 16;
__global__ void __launch_bounds__(SUM_BINS * SUM_RUNS)
    k_sum_spectra(const float2* __restrict__ part, long long units, int fft, float2* __restrict__ out) {
    __shared__ float2 red[SUM_RUNS][SUM_BINS];
    const int b = threadIdx.x % SUM_BINS, r = threadIdx.x / SUM_BINS;
    const int k = blockIdx.x * SUM_BINS + b;  // fft is a multiple of SUM_BINS
    const long long run = (units + SUM_RUNS - 1) / SUM_RUNS, u0 = r * run;
    const long long u1 = u0 + run < units ? u0 + run : units;
    float2 s = make_float2(0.f, 0.f);
    for (long long u = u0; u < u1; ++u) s = cadd(s, part[u * fft + k]);
    red[r][b] = s;
    __syncthreads();
    if (r != 0) return;
    float2 tot = make_float2(0.f, 0.f);
    for (int q = 0; q < SUM_RUNS; ++q) tot = cadd(tot, red[q][b]);
    out[k] = tot;
}

// dh[k] = Re IFFT(S)[k], k < K (one line), S_k = (P_k + conj P_{-k}) / 2 the
// Hermitian part of the summed pair spectra P (k_conv_bwd)
template <int FFT>
__global__ void __launch_bounds__(ConvGeom<FFT>::T) k_dh_finish(const float2* __restrict__ D, const float2* __restrict__ tw,
                                                                int K, float* __restrict__ dh) {
    constexpr int T = ConvGeom<FFT>::T;
    extern __shared__ __align__(16) float2 smem[];
    const int t = threadIdx.x;
    float2 v[CONV_E];
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) {
        const int k = t + m * T;
        const float2 a = D[k], b = D[(FFT - k) & (FFT - 1)];
        v[m] = cconj(make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y)));
    }
    fft_regs<FFT, CONV_E, (T <= 32)>(v, t, PadLine{smem}, tw);
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) {
        const int k = t + m * T;
        if (k < K) dh[k] = v[m].x / (float)FFT;
    }
}

// Correlator.cross: out = Re IFFT(FFT(a) conj(FFT(b))), a and b real,
// zero-padded / truncated to FFT; both travel in one complex line.
template <int FFT>
__global__ void __launch_bounds__(ConvGeom<FFT>::T) k_corr(const float* __restrict__ a, long long na,
                                                           const float* __restrict__ b, long long nb,
                                                           const float2* __restrict__ tw, float* __restrict__ out) {
    constexpr int T = ConvGeom<FFT>::T;
    constexpr bool WS = (T <= 32);
    extern __shared__ __align__(16) float2 smem[];
    const PadLine buf{smem};
    const int t = threadIdx.x;
    float2 v[CONV_E];
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) {
        const int i = t + m * T;
        v[m] = make_float2(i < na ? a[i] : 0.f, i < nb ? b[i] : 0.f);
    }
    fft_regs<FFT, CONV_E, WS>(v, t, buf, tw);
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) buf[t + m * T] = v[m];
    line_sync<WS>();
    float2 w[CONV_E];
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) {
        const int k = t + m * T;
        const float2 zc = cconj(buf[(FFT - k) & (FFT - 1)]);
        const float2 Ak = make_float2(0.5f * (v[m].x + zc.x), 0.5f * (v[m].y + zc.y));
        const float2 dZ = make_float2(0.5f * (v[m].x - zc.x), 0.5f * (v[m].y - zc.y));
        const float2 Bk = make_float2(dZ.y, -dZ.x);
        w[m] = cconj(cmul(Ak, cconj(Bk)));  // conj for the inverse
    }
    line_sync<WS>();
    fft_regs<FFT, CONV_E, WS>(w, t, buf, tw);
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) out[t + m * T] = w[m].x / (float)FFT;
}

// FFTAnalyzer.analyze: spectrum = FFT(samples[off + i] * window[i]) (real in)
template <int FFT>
__global__ void __launch_bounds__(ConvGeom<FFT>::T) k_analyze(const float* __restrict__ s, const float* __restrict__ w,
                                                              const float2* __restrict__ tw, float2* __restrict__ out) {
    constexpr int T = ConvGeom<FFT>::T;
    extern __shared__ __align__(16) float2 smem[];
    const int t = threadIdx.x;
    float2 v[CONV_E];
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) {
        const int i = t + m * T;
        v[m] = make_float2(s[i] * w[i], 0.f);
    }
    fft_regs<FFT, CONV_E, (T <= 32)>(v, t, PadLine{smem}, tw);
#pragma unroll
    for (int m = 0; m < CONV_E; ++m) out[t + m * T] = v[m];
}

// ---- host-side dispatch over the supported sizes ---------------------------

struct LineKernels {
    int fft;
    int threads, lines, smem, line_smem;
    cudaError_t (*prepare)();
    bool acc_smem;
    bool stash_smem;  // backward: Z stash in shared memory (else a global row per walker)
    void (*fwd)(dim3, int, cudaStream_t, const float*, long long, float*, long long, const float2*, const float2*, int,
                long long, long long, int, float*);
    void (*bwd)(dim3, int, cudaStream_t, const float*, long long, const float*, long long, const float2*,
                const float2*, int, long long, long long, float*, float2*, float2*);
    void (*dh)(cudaStream_t, const float2*, const float2*, int, float*);
    void (*corr)(cudaStream_t, const float*, long long, const float*, long long, const float2*, float*);
    void (*analyze)(cudaStream_t, const float*, const float*, const float2*, float2*);
};

template <int FFT>
cudaError_t prep_line() {
    using G = ConvGeom<FFT>;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_conv_fwd<FFT>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES))) return e;
    if ((e = cudaFuncSetAttribute(k_conv_bwd<FFT>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES_BWD))) return e;
    const int ls = spad_size(FFT) * 8;
    if ((e = cudaFuncSetAttribute(k_dh_finish<FFT>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls))) return e;
    if ((e = cudaFuncSetAttribute(k_corr<FFT>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls))) return e;
    return cudaFuncSetAttribute(k_analyze<FFT>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls);
}

template <int FFT>
void l_fwd(dim3 grid, int smem, cudaStream_t s, const float* x, long long nx, float* y, long long ny, const float2* H,
           const float2* tw, int hop, long long npairs, long long ppu, int warm, float* accg) {
    k_conv_fwd<FFT><<<grid, ConvGeom<FFT>::THREADS, smem, s>>>(x, nx, y, ny, H, tw, hop, npairs, ppu, warm, accg);
}
template <int FFT>
void l_bwd(dim3 grid, int, cudaStream_t s, const float* x, long long nx, const float* g, long long ny,
           const float2* H, const float2* tw, int hop, long long nblocks, long long bpu, float* dx, float2* part,
           float2* zs) {
    k_conv_bwd<FFT><<<grid, ConvGeom<FFT>::THREADS, ConvGeom<FFT>::SMEM_BYTES_BWD, s>>>(x, nx, g, ny, H, tw, hop,
                                                                                     nblocks, bpu, dx, part, zs);
}
template <int FFT>
void l_dh(cudaStream_t s, const float2* D, const float2* tw, int K, float* dh) {
    k_dh_finish<FFT><<<1, ConvGeom<FFT>::T, spad_size(FFT) * 8, s>>>(D, tw, K, dh);
}
template <int FFT>
void l_corr(cudaStream_t s, const float* a, long long na, const float* b, long long nb, const float2* tw, float* out) {
    k_corr<FFT><<<1, ConvGeom<FFT>::T, spad_size(FFT) * 8, s>>>(a, na, b, nb, tw, out);
}
template <int FFT>
void l_an(cudaStream_t s, const float* smp, const float* w, const float2* tw, float2* out) {
    k_analyze<FFT><<<1, ConvGeom<FFT>::T, spad_size(FFT) * 8, s>>>(smp, w, tw, out);
}

#define MFFT_LINEK(F)                                                                                       \
    {F,           ConvGeom<F>::THREADS, ConvGeom<F>::LINES, ConvGeom<F>::SMEM_BYTES, spad_size(F) * 8,     \
     &prep_line<F>, ConvGeom<F>::ACC_SMEM, ConvGeom<F>::STASH, &l_fwd<F>, &l_bwd<F>, &l_dh<F>, &l_corr<F>,     \
     &l_an<F>}

const LineKernels g_linek[] = {MFFT_LINEK(64),   MFFT_LINEK(128),  MFFT_LINEK(256),
                               MFFT_LINEK(512),  MFFT_LINEK(1024), MFFT_LINEK(2048),
                               MFFT_LINEK(4096), MFFT_LINEK(8192), MFFT_LINEK(16384)};

const LineKernels* find_linek(int fft) {
    for (const auto& k : g_linek)
        if (k.fft == fft) return &k;
    return nullptr;
}

}  // namespace

}  // namespace mfft

using namespace mfft;

// ---------------------------------------------------------------------------
// Convolver
// ---------------------------------------------------------------------------

static const BatchedKernel* e16_kernel(int n) {
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    for (int i = 0; i < cnt; ++i)
        if (ks[i].n == n && ks[i].e == 16) return &ks[i];
    return nullptr;
}

struct mfft_conv {
    mfft_ctx* ctx = nullptr;
    int64_t fft = 0, K = 0, hop = 0;
    const LineKernels* lk = nullptr;
    float2* tw = nullptr;    // line twiddles (context-owned)
    float2* H = nullptr;     // kernel spectrum, natural order
    float2* part = nullptr;  // dh partial spectra, units x fft
    float2* Dsum = nullptr;
    long long part_units = 0;
    float* accg = nullptr;   // forward overlap accumulators when not in smem
    long long accg_units = 0;
    int precision = MFFT_CONV_FLOAT32;  // forward arithmetic (FusedConvolver.Precision)
    int fp16_occ = 0;                   // resident CTAs per SM of the FP16 forward kernel
};

static int conv_units(mfft_conv* c, long long work, long long* per_unit, long long* units, int per_sm = 2) {
    // enough walkers to fill the GPU, a few block pairs each
    const long long lines = c->lk->lines;
    long long want = (long long)c->ctx->sms * per_sm * lines;
    if (want > work) want = work;
    if (want < 1) want = 1;
    *per_unit = (work + want - 1) / want;
    *units = (work + *per_unit - 1) / *per_unit;
    return MFFT_SUCCESS;
}

extern "C" int mfft_conv_create(mfft_ctx* ctx, const float* kernel, int64_t kernel_len, int64_t fft_size,
                                mfft_conv** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    *out = nullptr;
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    if (!is_pow2_in(fft_size, 64, MFFT_MAX_SINGLE_N))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, fft_size, -1, -1,
                         "Unsupported FFT size: %lld. The convolver takes powers of two 64..16384",
                         (long long)fft_size);
    if (kernel_len < 1 || kernel_len >= fft_size || !kernel)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1,
                         "fftSize must be > kernel.count; got fftSize=%lld, kernel.count=%lld", (long long)fft_size,
                         (long long)kernel_len);
    DeviceGuard g(ctx->device);
    mfft_conv* c = new mfft_conv();
    c->ctx = ctx;
    c->fft = fft_size;
    c->K = kernel_len;
    c->hop = fft_size - kernel_len + 1;
    c->lk = find_linek((int)fft_size);
    // the kernel spectrum is computed with the context's batched kernel for
    // this size; its twiddle rows (E = 16) are the ones the line kernels use
    BatchedBinding spec;
    const BatchedKernel* bk = e16_kernel((int)fft_size);
    int st = bind_batched(ctx, bk, &spec);
    c->tw = spec.tw;
    cudaError_t e = cudaSuccess;
    if (!st) e = c->lk->prepare();
    if (!st && e != cudaSuccess) st = cuda_error(e, "convolver kernel attributes");
    if (!st) {
        e = cudaMalloc(&c->H, sizeof(float2) * fft_size * 2);
        if (e != cudaSuccess) st = set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "kernel spectrum: %s", cudaGetErrorString(e));
    }
    if (!st) {
        // kernel spectrum = FFT(h zero-padded) (Convolve.swift:27-31), on the device
        c->Dsum = c->H + fft_size;
        std::vector<float2> hk((size_t)fft_size, make_float2(0.f, 0.f));
        for (int64_t i = 0; i < kernel_len; ++i) hk[i].x = kernel[i];
        e = cudaMemcpyAsync(c->Dsum, hk.data(), sizeof(float2) * fft_size, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) st = cuda_error(e, "kernel upload");
        if (!st) {
            e = bk->fwd(c->Dsum, c->H, 1, c->tw, ctx->dev_err, ctx->stream, 0);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) st = cuda_error(e, "kernel spectrum");
        }
    }
    if (st) {
        mfft_conv_destroy(c);
        return st;
    }
    *out = c;
    return MFFT_SUCCESS;
}

extern "C" int mfft_conv_destroy(mfft_conv* c) {
    if (!c) return MFFT_SUCCESS;
    DeviceGuard g(c->ctx->device);
    cudaFree(c->H);
    cudaFree(c->part);
    cudaFree(c->accg);
    delete c;
    return MFFT_SUCCESS;
}

extern "C" int64_t mfft_conv_block_size(const mfft_conv* c) { return c ? c->fft : 0; }
extern "C" int64_t mfft_conv_hop_size(const mfft_conv* c) { return c ? c->hop : 0; }
extern "C" int64_t mfft_conv_kernel_len(const mfft_conv* c) { return c ? c->K : 0; }

extern "C" int mfft_conv_set_precision(mfft_conv* c, int precision) {
    if (!c) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "convolver is NULL");
    if (precision < MFFT_CONV_FLOAT32 || precision > MFFT_CONV_FP16_MIXED)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, precision, -1, "unknown precision %d", precision);
    if (precision != MFFT_CONV_FLOAT32) {
        if (c->fft != 4096)  // FusedConvolver.swift:19, 56-57
            return set_error(MFFT_ERR_INVALID_ARGUMENT, 4096, c->fft, -1,
                             "FusedConvolver only supports fftSize=4096 in FP16 modes, got %lld", (long long)c->fft);
        DeviceGuard g(c->ctx->device);
        const int occ = conv_fp16_ctas_per_sm(precision);
        if (occ <= 0) {
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_error(e, "FP16 convolver kernel attributes");
            return set_error(MFFT_ERR_LIBRARY_BUILD, -1, -1, -1, "the FP16 convolver kernel cannot be resident on this device");
        }
        c->fp16_occ = occ;
    }
    c->precision = precision;
    return MFFT_SUCCESS;
}

static int conv_fwd_device(mfft_conv* c, const float* x, long long nx, float* y, cudaStream_t s) {
    const long long ny = nx + c->K - 1;
    const long long nout = (ny + c->hop - 1) / c->hop;  // output blocks (virtual zeros past nx)
    const long long npairs = (nout + 1) / 2;
    long long ppu, units;
    const int warm = (int)((c->fft - 1) / c->hop);  // earlier blocks overlapping a range start
    if (c->precision != MFFT_CONV_FLOAT32) {  // one walker per CTA, as many as are resident
        conv_units(c, npairs, &ppu, &units, c->fp16_occ);
        cudaError_t e = conv_fp16_forward(c->precision, units, s, x, nx, y, ny, c->H, c->tw, (int)c->hop, npairs,
                                          ppu, warm);
        return e == cudaSuccess ? MFFT_SUCCESS : cuda_error(e, "FP16 convolver launch");
    }
    conv_units(c, npairs, &ppu, &units);
    const long long ctas = (units + c->lk->lines - 1) / c->lk->lines;
    if (!c->lk->acc_smem && ctas * c->lk->lines > c->accg_units) {
        cudaFree(c->accg);
        c->accg = nullptr;
        c->accg_units = 0;
        cudaError_t e = cudaMalloc(&c->accg, sizeof(float) * 2 * c->fft * ctas * c->lk->lines);
        if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "overlap accumulators: %s", cudaGetErrorString(e));
        c->accg_units = ctas * c->lk->lines;
    }
    c->lk->fwd(dim3((unsigned)ctas), c->lk->smem, s, x, nx, y, ny, c->H, c->tw, (int)c->hop, npairs, ppu, warm,
               c->accg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "convolver launch");
    return MFFT_SUCCESS;
}

extern "C" int mfft_conv_apply(mfft_conv* c, const float* signal, int64_t n, float* out, int flags, void* stream) {
    if (!c) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "convolver is NULL");
    if (n < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, n, -1, "signal length must be >= 0");
    if (flags != MFFT_HOST_MEMORY && flags != MFFT_DEVICE_MEMORY)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown flags %d", flags);
    if (!out || (n > 0 && !signal)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL buffer");
    DeviceGuard g(c->ctx->device);
    if (flags == MFFT_DEVICE_MEMORY) return conv_fwd_device(c, signal, n, out, (cudaStream_t)stream);
    const size_t in_b = (size_t)n * 4, out_b = (size_t)(n + c->K - 1) * 4;
    return run_host_staged(c->ctx, signal, out, in_b, out_b, [&](void* di, void* dout, cudaStream_t s) {
        return conv_fwd_device(c, (const float*)di, n, (float*)dout, s);
    });
}

static int conv_bwd_device(mfft_conv* c, const float* x, long long nx, const float* gy, float* dx, float* dh,
                           cudaStream_t s) {
    const long long ny = nx + c->K - 1;
    const long long nblocks = (nx + c->hop - 1) / c->hop;
    long long bpu = 1, units = 1;
    if (nblocks > 0) conv_units(c, nblocks, &bpu, &units);
    if (bpu % 2) ++bpu;  // blocks go in pairs through one inverse
    units = nblocks > 0 ? (nblocks + bpu - 1) / bpu : 1;
    const long long ctas = (units + c->lk->lines - 1) / c->lk->lines;
    const long long slots = ctas * c->lk->lines;
    // rows of partial spectra, then (when shared memory cannot hold it) one
    // Z stash row per walker
    const long long rows = c->lk->stash_smem ? slots : 2 * slots;
    if (rows > c->part_units) {
        if (c->part) cudaFree(c->part);
        c->part = nullptr;
        c->part_units = 0;
        cudaError_t e = cudaMalloc(&c->part, sizeof(float2) * c->fft * rows);
        if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "dh partials: %s", cudaGetErrorString(e));
        c->part_units = rows;
    }
    float2* zs = c->lk->stash_smem ? nullptr : c->part + slots * c->fft;
    c->lk->bwd(dim3((unsigned)ctas), c->lk->smem, s, x, nx, gy, ny, c->H, c->tw, (int)c->hop, nblocks, bpu, dx,
               c->part, zs);
    if (dh) {
        k_sum_spectra<<<(unsigned)(c->fft / SUM_BINS), SUM_BINS * SUM_RUNS, 0, s>>>(c->part, slots, (int)c->fft,
                                                                                 c->Dsum);
        c->lk->dh(s, c->Dsum, c->tw, (int)c->K, dh);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "convolver backward launch");
    return MFFT_SUCCESS;
}

extern "C" int mfft_conv_backward(mfft_conv* c, const float* signal, int64_t n, const float* grad_out,
                                  float* grad_signal, float* grad_kernel, int flags, void* stream) {
    if (!c) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "convolver is NULL");
    if (n < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, n, -1, "signal length must be >= 0");
    if (flags != MFFT_HOST_MEMORY && flags != MFFT_DEVICE_MEMORY)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown flags %d", flags);
    if (!grad_out || (n > 0 && !signal)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL buffer");
    if (!grad_signal && !grad_kernel) return MFFT_SUCCESS;
    DeviceGuard g(c->ctx->device);
    const long long ny = n + c->K - 1;
    if (flags == MFFT_DEVICE_MEMORY) {
        if (!grad_signal && n > 0)
            return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "device calls need grad_signal storage");
        return conv_bwd_device(c, signal, n, grad_out, grad_signal, grad_kernel, (cudaStream_t)stream);
    }
    // host arrays: [x | g] in, [dx | dh] out
    const size_t xin = (size_t)n * 4, gin = (size_t)ny * 4;
    const size_t dxo = (size_t)n * 4, dho = (size_t)c->K * 4;
    std::vector<float> hin(n + ny), hout(n + c->K);
    if (n) memcpy(hin.data(), signal, xin);
    memcpy(hin.data() + n, grad_out, gin);
    int st = run_host_staged(c->ctx, hin.data(), hout.data(), xin + gin, dxo + dho,
                             [&](void* di, void* dout, cudaStream_t s) {
                                 const float* dxi = (const float*)di;
                                 float* o = (float*)dout;
                                 return conv_bwd_device(c, dxi, n, dxi + n, o, o + n, s);
                             });
    if (st) return st;
    if (grad_signal && n) memcpy(grad_signal, hout.data(), dxo);
    if (grad_kernel) memcpy(grad_kernel, hout.data() + n, dho);
    return MFFT_SUCCESS;
}

// ---------------------------------------------------------------------------
// Correlator
// ---------------------------------------------------------------------------

struct mfft_corr {
    mfft_ctx* ctx = nullptr;
    int64_t fft = 0;
    const LineKernels* lk = nullptr;
    float2* tw = nullptr;
};

extern "C" int mfft_corr_create(mfft_ctx* ctx, int64_t fft_size, mfft_corr** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    *out = nullptr;
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    if (!is_pow2_in(fft_size, 64, MFFT_MAX_SINGLE_N))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, fft_size, -1, -1,
                         "Unsupported FFT size: %lld. Supported: powers of two 64..16384", (long long)fft_size);
    DeviceGuard g(ctx->device);
    mfft_corr* c = new mfft_corr();
    c->ctx = ctx;
    c->fft = fft_size;
    c->lk = find_linek((int)fft_size);
    int st = ctx_twiddles(ctx, e16_kernel((int)fft_size), &c->tw);
    if (!st) {
        cudaError_t e = c->lk->prepare();
        if (e != cudaSuccess) st = cuda_error(e, "correlator kernel attributes");
    }
    if (st) {
        delete c;
        return st;
    }
    *out = c;
    return MFFT_SUCCESS;
}

extern "C" int mfft_corr_destroy(mfft_corr* c) {
    delete c;
    return MFFT_SUCCESS;
}

extern "C" int mfft_corr_cross(mfft_corr* c, const float* a, int64_t na, const float* b, int64_t nb, float* out,
                               int flags, void* stream) {
    if (!c) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "correlator is NULL");
    if (na < 0 || nb < 0) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "negative length");
    if (!out || (na && !a) || (nb && !b)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL buffer");
    if (flags != MFFT_HOST_MEMORY && flags != MFFT_DEVICE_MEMORY)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown flags %d", flags);
    DeviceGuard g(c->ctx->device);
    const int64_t ua = na < c->fft ? na : c->fft, ub = nb < c->fft ? nb : c->fft;
    auto body = [&](const float* da, const float* db, float* dout, cudaStream_t s) {
        c->lk->corr(s, da, ua, db, ub, c->tw, dout);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(e, "correlator launch");
    };
    if (flags == MFFT_DEVICE_MEMORY) return body(a, b, out, (cudaStream_t)stream);
    std::vector<float> hin((size_t)(ua + ub) + 1);
    if (ua) memcpy(hin.data(), a, ua * 4);
    if (ub) memcpy(hin.data() + ua, b, ub * 4);
    return run_host_staged(c->ctx, hin.data(), out, (size_t)(ua + ub) * 4, (size_t)c->fft * 4,
                           [&](void* di, void* dout, cudaStream_t s) {
                               return body((const float*)di, (const float*)di + ua, (float*)dout, s);
                           });
}

// ---------------------------------------------------------------------------
// windows and FFTAnalyzer
// ---------------------------------------------------------------------------

static double bessel_i0(double x) {
    double result = 1.0, term = 1.0, hx = x / 2.0;
    for (int k = 1; k <= 30; ++k) {
        term *= (hx * hx) / (double)(k * k);
        result += term;
        if (term < 1e-12 * result) break;
    }
    return result;
}

// WindowType.coefficients (Window.swift:12-95); the vDSP windows use the
// definitions of Apple's vDSP reference (full window, denominator N):
// Hann NORM 0.8165*(1 - cos 2*pi*n/N), Hamming 0.54 - 0.46 cos, Blackman
// 0.42 - 0.5 cos + 0.08 cos(2x).
extern "C" int mfft_window(int kind, int64_t n, double beta, float* out) {
    if (n < 0 || (n > 0 && !out)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "bad window arguments");
    if (kind < MFFT_WINDOW_HANN || kind > MFFT_WINDOW_RECTANGULAR)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown window kind %d", kind);
    const double pi = 3.14159265358979323846;
    for (int64_t k = 0; k < n; ++k) {
        const double x = 2.0 * pi * (double)k / (double)n;
        double w = 1.0;
        switch (kind) {
            case MFFT_WINDOW_HANN: w = 0.8165 * (1.0 - cos(x)); break;
            case MFFT_WINDOW_HAMMING: w = 0.54 - 0.46 * cos(x); break;
            case MFFT_WINDOW_BLACKMAN: w = 0.42 - 0.5 * cos(x) + 0.08 * cos(2.0 * x); break;
            case MFFT_WINDOW_FLAT_TOP:
                w = 0.21557895 - 0.41663158 * cos(x) + 0.277263158 * cos(2.0 * x) - 0.083578947 * cos(3.0 * x) +
                    0.006947368 * cos(4.0 * x);
                break;
            case MFFT_WINDOW_KAISER: {
                const double half = (double)(n - 1) / 2.0;
                const double t = half > 0 ? ((double)k - half) / half : 0.0;
                const double v = 1.0 - t * t;
                w = bessel_i0(beta * sqrt(v > 0 ? v : 0.0)) / bessel_i0(beta);
                break;
            }
            default: w = 1.0;
        }
        out[k] = (float)w;
    }
    return MFFT_SUCCESS;
}

struct mfft_analyzer {
    mfft_ctx* ctx = nullptr;
    int64_t size = 0;
    double sample_rate = 0;
    const LineKernels* lk = nullptr;
    float2* tw = nullptr;
    float* window = nullptr;  // device
};

extern "C" int mfft_analyzer_create(mfft_ctx* ctx, int64_t size, double sample_rate, int window_kind,
                                    double kaiser_beta, mfft_analyzer** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    *out = nullptr;
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    if (!is_pow2_in(size, 64, MFFT_MAX_SINGLE_N))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, size, -1, -1,
                         "Unsupported FFT size: %lld. Supported: powers of two 64..16384", (long long)size);
    std::vector<float> w((size_t)size);
    int st = mfft_window(window_kind, size, kaiser_beta, w.data());
    if (st) return st;
    DeviceGuard g(ctx->device);
    mfft_analyzer* a = new mfft_analyzer();
    a->ctx = ctx;
    a->size = size;
    a->sample_rate = sample_rate;
    a->lk = find_linek((int)size);
    st = ctx_twiddles(ctx, e16_kernel((int)size), &a->tw);
    cudaError_t e = cudaSuccess;
    if (!st) e = a->lk->prepare();
    if (!st && e != cudaSuccess) st = cuda_error(e, "analyzer kernel attributes");
    if (!st) {
        e = cudaMalloc(&a->window, sizeof(float) * size);
        if (e == cudaSuccess) e = cudaMemcpy(a->window, w.data(), sizeof(float) * size, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "window: %s", cudaGetErrorString(e));
    }
    if (st) {
        mfft_analyzer_destroy(a);
        return st;
    }
    *out = a;
    return MFFT_SUCCESS;
}

extern "C" int mfft_analyzer_destroy(mfft_analyzer* a) {
    if (!a) return MFFT_SUCCESS;
    DeviceGuard g(a->ctx->device);
    cudaFree(a->window);
    delete a;
    return MFFT_SUCCESS;
}

extern "C" int mfft_analyzer_analyze(mfft_analyzer* a, const float* samples, int64_t count, int64_t offset,
                                     void* spectrum, int flags, void* stream) {
    if (!a) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "analyzer is NULL");
    if (offset < 0 || count < 0 || offset + a->size > count)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1,
                         "offset + size <= samples.count required (offset %lld, size %lld, count %lld)",
                         (long long)offset, (long long)a->size, (long long)count);
    if (!samples || !spectrum) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL buffer");
    if (flags != MFFT_HOST_MEMORY && flags != MFFT_DEVICE_MEMORY)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "unknown flags %d", flags);
    DeviceGuard g(a->ctx->device);
    auto body = [&](const float* s_, float2* o, cudaStream_t s) {
        a->lk->analyze(s, s_, a->window, a->tw, o);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(e, "analyzer launch");
    };
    if (flags == MFFT_DEVICE_MEMORY) return body(samples + offset, (float2*)spectrum, (cudaStream_t)stream);
    return run_host_staged(a->ctx, samples + offset, spectrum, (size_t)a->size * 4, (size_t)a->size * 8,
                           [&](void* di, void* dout, cudaStream_t s) { return body((const float*)di, (float2*)dout, s); });
}
