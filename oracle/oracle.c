/*
 * oracle.c -- CPU oracle for the MetalFFT batched complex FFT path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this file.  It is used by tests/ (as the checker), by
 * __graft_entry__.smoke() (as the checker) and by bench.py's CPU-baseline leg
 * (timed beside the GPU, never as the thing measured on the GPU).
 *
 * Two families live here:
 *
 *  1. FP64 ground truth ("mfo_*_c128"): an iterative radix-2 FFT and a naive
 *     O(N^2) DFT with exact integer angle reduction.  The DFT pins the FFT;
 *     the test suite pins both against the reference's own known-answer tests
 *     (impulse -> all ones, cosine peak bin, DFT8 matrix entries, CT twiddle
 *     table) and against numpy's pocketfft, the stand-in for the reference's
 *     comparison path Apple vDSP (vDSP_fft_zop, macOS system framework, no
 *     version pin; call sites Tests/MetalFFTTests/MetalFFTTests.swift:164-188).
 *
 *  2. FP32 restatement of the reference's CPU-visible algorithm ("mfo_ref_*"):
 *     the radix-4 (+ trailing radix-2) Stockham passes of
 *     Sources/MetalFFT/Resources/fft_multisize.metal:25-55,62-687 with one
 *     sincos per butterfly and w2 = w1^2, w3 = w2*w1; the four-step plan of
 *     Sources/MetalFFT/FFT/MetalFFT.swift:206-277 with the splits of
 *     Sources/MetalFFT/Internal/MetalContext.swift:57-66 (8192 = 64x128,
 *     16384 = 128x128, extended here to 2^m = 2^floor(m/2) x 2^ceil(m/2) up to
 *     2^20); the conjugate-trick inverse of MetalFFT.swift:56-65; the
 *     overlap-add Convolver of Sources/MetalFFT/DSP/Convolve.swift:19-76; the
 *     Correlator of Sources/MetalFFT/DSP/Correlate.swift:31-61.  These are
 *     parallel over independent transforms / blocks with OpenMP and serve as
 *     the timed CPU baseline (the reference's own CPU comparison path is
 *     Accelerate, which does not exist on Linux).
 *
 * Layout everywhere: interleaved complex (re, im), transform b at offset b*n.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MFO_PI 3.14159265358979323846

static int mfo_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    return nthreads;
#else
    (void)nthreads;
    return 1;
#endif
}

int mfo_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static int ilog2_i64(int64_t n) {
    int l = 0;
    while (((int64_t)1 << l) < n) ++l;
    return l;
}

/* ------------------------------------------------------------------------ */
/* FP64 ground truth                                                         */
/* ------------------------------------------------------------------------ */

/* exp(sign * 2*pi*i * m / n) in FP64 with the index reduced exactly first. */
static void root64(int64_t m, int64_t n, int sign, double* c, double* s) {
    m %= n;
    if (m < 0) m += n;
    double a = 2.0 * MFO_PI * (double)m / (double)n;
    *c = cos(a);
    *s = (double)sign * sin(a);
}

/* Naive DFT: X[k] = sum_j x[j] exp(sign*2*pi*i*j*k/n).  O(n^2); small n only. */
void mfo_dft_c128(const double* in, double* out, int64_t n, int sign) {
    double* tw = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    for (int64_t m = 0; m < n; ++m) root64(m, n, sign, &tw[2 * m], &tw[2 * m + 1]);
    for (int64_t k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            int64_t m = (j * k) % n;
            double xr = in[2 * j], xi = in[2 * j + 1];
            double wr = tw[2 * m], wi = tw[2 * m + 1];
            sr += xr * wr - xi * wi;
            si += xr * wi + xi * wr;
        }
        out[2 * k] = sr;
        out[2 * k + 1] = si;
    }
    free(tw);
}

/* One FP64 radix-2 Stockham FFT of length n (power of two), unscaled.
 * work: 2*n doubles of scratch.  tw: n/2 roots exp(sign*2*pi*i*m/n). */
static void fft64_one(const double* in, double* out, double* work, const double* tw,
                      int64_t n) {
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    int L = ilog2_i64(n);
    const double* src = in;
    double* bufs[2];
    /* Choose ping-pong so that the final pass lands in `out`. */
    bufs[(L - 1) & 1] = out;
    bufs[L & 1] = work;
    int64_t half = n / 2;
    int64_t ns = 1;
    for (int p = 0; p < L; ++p) {
        double* dst = bufs[p & 1];
        if (p == L - 1) dst = out;
        for (int64_t j = 0; j < half; ++j) {
            int64_t k = j & (ns - 1);
            /* twiddle exp(sign*2*pi*i*k/(2*ns)) = tw[k * (n/(2*ns))] */
            int64_t ti = k * (n / (2 * ns));
            double wr = tw[2 * ti], wi = tw[2 * ti + 1];
            double ar = src[2 * j], ai = src[2 * j + 1];
            double br = src[2 * (j + half)], bi = src[2 * (j + half) + 1];
            double tr = br * wr - bi * wi, tii = br * wi + bi * wr;
            int64_t d = (j - k) * 2 + k; /* expand(j, ns, 2) */
            dst[2 * d] = ar + tr;
            dst[2 * d + 1] = ai + tii;
            dst[2 * (d + ns)] = ar - tr;
            dst[2 * (d + ns) + 1] = ai - tii;
        }
        src = dst;
        ns *= 2;
    }
}

/* Batched FP64 FFT, unscaled.  sign=-1 is the forward DFT convention of
 * fft_multisize.metal:70 (TWO_PI_OVER_N = -2*pi/N). */
void mfo_fft_c128(const double* in, double* out, int64_t n, int64_t batch, int sign,
                  int nthreads) {
    double* tw = (double*)malloc(sizeof(double) * 2 * (size_t)(n / 2 + 1));
    for (int64_t m = 0; m < n / 2 + 1; ++m) root64(m, n, sign, &tw[2 * m], &tw[2 * m + 1]);
    int nt = mfo_set_threads(nthreads);
#pragma omp parallel num_threads(nt)
    {
        double* work = (double*)malloc(sizeof(double) * 2 * (size_t)n);
        double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)n);
#pragma omp for schedule(static)
        for (int64_t b = 0; b < batch; ++b) {
            const double* x = in + 2 * n * b;
            double* y = out + 2 * n * b;
            if (x == y) {
                memcpy(tmp, x, sizeof(double) * 2 * (size_t)n);
                fft64_one(tmp, y, work, tw, n);
            } else {
                fft64_one(x, y, work, tw, n);
            }
        }
        free(work);
        free(tmp);
    }
    free(tw);
}

/* Complex64 (float) in -> FP64 FFT -> complex128 out.  Used to compute the
 * ground truth of a float input without an extra conversion pass in Python. */
void mfo_fft_c64_to_c128(const float* in, double* out, int64_t n, int64_t batch, int sign,
                         int nthreads) {
    int nt = mfo_set_threads(nthreads);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < 2 * n * batch; ++i) out[i] = (double)in[i];
    mfo_fft_c128(out, out, n, batch, sign, nthreads);
}

/* Relative RMS error ||y - ref|| / ||ref|| accumulated in FP64
 * (the L2 definition of Tests/MetalFFTTests/MetalFFTTests.swift:190-198). */
double mfo_rel_rms_c64_vs_c128(const float* y, const double* ref, int64_t count_complex,
                               int nthreads) {
    double num = 0.0, den = 0.0;
    int nt = mfo_set_threads(nthreads);
#pragma omp parallel for num_threads(nt) reduction(+ : num, den) schedule(static)
    for (int64_t i = 0; i < 2 * count_complex; ++i) {
        double d = (double)y[i] - ref[i];
        num += d * d;
        den += ref[i] * ref[i];
    }
    return den > 0.0 ? sqrt(num / den) : sqrt(num);
}

/* ------------------------------------------------------------------------ */
/* FP32 restatement of the reference path                                   */
/* ------------------------------------------------------------------------ */

typedef struct {
    float x, y;
} c32;

static inline c32 cmul32(c32 a, c32 b) {
    c32 r = {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
    return r;
}
static inline c32 cadd32(c32 a, c32 b) {
    c32 r = {a.x + b.x, a.y + b.y};
    return r;
}
static inline c32 csub32(c32 a, c32 b) {
    c32 r = {a.x - b.x, a.y - b.y};
    return r;
}

/* Radix-4 DIT butterfly, forward sign (fft_multisize.metal:29-40 semantics). */
static inline void radix4_32(c32* x0, c32* x1, c32* x2, c32* x3) {
    c32 t0 = cadd32(*x0, *x2), t1 = cadd32(*x1, *x3);
    c32 t2 = csub32(*x0, *x2), t3 = csub32(*x1, *x3);
    c32 t3r = {t3.y, -t3.x}; /* -i * t3 */
    *x0 = cadd32(t0, t1);
    *x1 = cadd32(t2, t3r);
    *x2 = csub32(t0, t1);
    *x3 = csub32(t2, t3r);
}

/* One length-n forward FFT (n = 4^a * 2^b, b in {0,1}) as the reference's
 * in-threadgroup Stockham: passes of radix 4 with stride 4^p, a trailing
 * radix-2 pass when log2(n) is odd.  Twiddle per butterfly position `pos`:
 * one sincos of (-2*pi/n)*pos*(n/(R*stride)) in FP32, w2=w1^2, w3=w2*w1
 * (fft_multisize.metal:48-55,100-102; radix-2 tail :252-280). */
static void ref_stockham_one(const c32* in, c32* out, c32* b0, c32* b1, int n) {
    const float two_pi_over_n = -2.0f * (float)MFO_PI / (float)n;
    int L = ilog2_i64(n);
    int n4 = L / 2;          /* radix-4 passes */
    int has2 = L & 1;        /* trailing radix-2 */
    int npass = n4 + has2;
    const c32* src = in;
    int stride = 1;
    for (int p = 0; p < npass; ++p) {
        int last = (p == npass - 1);
        c32* dst = last ? out : ((p & 1) ? b1 : b0);
        if (p < n4) {
            int T = n / 4;
            int twf = n / (4 * stride);
            for (int tid = 0; tid < T; ++tid) {
                int pos = tid & (stride - 1);
                int grp = tid / stride;
                c32 x0 = src[tid], x1 = src[tid + T], x2 = src[tid + 2 * T], x3 = src[tid + 3 * T];
                if (stride > 1) {
                    float a1 = two_pi_over_n * (float)(pos * twf);
                    c32 w1 = {cosf(a1), sinf(a1)};
                    c32 w2 = cmul32(w1, w1);
                    c32 w3 = cmul32(w2, w1);
                    x1 = cmul32(x1, w1);
                    x2 = cmul32(x2, w2);
                    x3 = cmul32(x3, w3);
                }
                radix4_32(&x0, &x1, &x2, &x3);
                int wr = grp * stride * 4 + pos;
                dst[wr] = x0;
                dst[wr + stride] = x1;
                dst[wr + 2 * stride] = x2;
                dst[wr + 3 * stride] = x3;
            }
            stride *= 4;
        } else {
            int T = n / 2;
            for (int tid = 0; tid < T; ++tid) {
                int pos = tid & (stride - 1);
                int grp = tid / stride;
                c32 x0 = src[tid], x1 = src[tid + T];
                float a1 = two_pi_over_n * (float)(pos * (n / (2 * stride)));
                c32 w1 = {cosf(a1), sinf(a1)};
                x1 = cmul32(x1, w1);
                int wr = grp * stride * 2 + pos;
                dst[wr] = cadd32(x0, x1);
                dst[wr + stride] = csub32(x0, x1);
            }
            stride *= 2;
        }
        src = dst;
    }
    if (npass == 0) out[0] = in[0];
}

/* Four-step plan of MetalFFT.swift:206-277 for one transform of n = n1*n2:
 * transpose (n2 x n1 -> n1 x n2), n1 FFTs of n2, twiddle W_n^{row*col} +
 * transpose (fft_multisize.metal:700-727), n2 FFTs of n1, transpose back. */
static void ref_fourstep_one(const c32* in, c32* out, c32* tA, c32* tB, c32* s0, c32* s1,
                             int n1, int n2) {
    int n = n1 * n2;
    /* step 0: in is n2 rows x n1 cols; tA is n1 x n2 */
    for (int r = 0; r < n2; ++r)
        for (int c = 0; c < n1; ++c) tA[c * n2 + r] = in[r * n1 + c];
    /* step 1: n1 rows of length n2 */
    for (int r = 0; r < n1; ++r) ref_stockham_one(tA + (size_t)r * n2, tB + (size_t)r * n2, s0, s1, n2);
    /* step 2: twiddle + transpose n1 x n2 -> n2 x n1 (FP32 angle, un-reduced,
     * as fft_multisize.metal:720) */
    for (int row = 0; row < n1; ++row)
        for (int col = 0; col < n2; ++col) {
            float ang = -2.0f * (float)MFO_PI * (float)(row * col) / (float)n;
            c32 w = {cosf(ang), sinf(ang)};
            tA[col * n1 + row] = cmul32(tB[row * n2 + col], w);
        }
    /* step 3: n2 rows of length n1 */
    for (int r = 0; r < n2; ++r) ref_stockham_one(tA + (size_t)r * n1, tB + (size_t)r * n1, s0, s1, n1);
    /* step 4: n2 x n1 -> n1 x n2 */
    for (int r = 0; r < n2; ++r)
        for (int c = 0; c < n1; ++c) out[c * n2 + r] = tB[r * n1 + c];
}

/* The reference descriptor's split of n into (n1, n2) for the four-step path
 * (MetalContext.swift:57-66), extended past 16384 with n1 = 2^floor(m/2). */
void mfo_ref_fourstep_split(int n, int* n1, int* n2) {
    if (n == 8192) {
        *n1 = 64;
        *n2 = 128;
        return;
    }
    int L = ilog2_i64(n);
    *n1 = 1 << (L / 2);
    *n2 = n / *n1;
}

/* Batched FP32 reference path.  inverse != 0 -> conj, forward, conj * 1/n
 * (MetalFFT.swift:56-65).  n in 64..2^20, power of two. */
void mfo_ref_fft_c64(const float* in, float* out, int n, int64_t batch, int inverse,
                     int nthreads) {
    int nt = mfo_set_threads(nthreads);
    int single = (n <= 4096);
    int n1 = 0, n2 = 0;
    if (!single) mfo_ref_fourstep_split(n, &n1, &n2);
#pragma omp parallel num_threads(nt)
    {
        c32* x = (c32*)malloc(sizeof(c32) * (size_t)n);
        c32* y = (c32*)malloc(sizeof(c32) * (size_t)n);
        c32* s0 = (c32*)malloc(sizeof(c32) * (size_t)n);
        c32* s1 = (c32*)malloc(sizeof(c32) * (size_t)n);
        c32* tA = single ? NULL : (c32*)malloc(sizeof(c32) * (size_t)n);
        c32* tB = single ? NULL : (c32*)malloc(sizeof(c32) * (size_t)n);
#pragma omp for schedule(static)
        for (int64_t b = 0; b < batch; ++b) {
            const c32* src = (const c32*)in + (size_t)n * b;
            c32* dst = (c32*)out + (size_t)n * b;
            for (int i = 0; i < n; ++i) {
                x[i] = src[i];
                if (inverse) x[i].y = -x[i].y;
            }
            if (single)
                ref_stockham_one(x, y, s0, s1, n);
            else
                ref_fourstep_one(x, y, tA, tB, s0, s1, n1, n2);
            if (inverse) {
                float inv = 1.0f / (float)n;
                for (int i = 0; i < n; ++i) {
                    dst[i].x = y[i].x * inv;
                    dst[i].y = -y[i].y * inv;
                }
            } else {
                memcpy(dst, y, sizeof(c32) * (size_t)n);
            }
        }
        free(x);
        free(y);
        free(s0);
        free(s1);
        free(tA);
        free(tB);
    }
}

/* ------------------------------------------------------------------------ */
/* Convolver / Correlator                                                   */
/* ------------------------------------------------------------------------ */

/* Overlap-add linear convolution, FP32 restatement of Convolve.swift:19-76:
 * hop = fft - K + 1, kernel spectrum = FFT(h zero-padded), per block
 * FFT -> * H -> inverse (conj trick) -> add real parts.  y has nx + K - 1
 * samples.  Blocks that do not overlap run in parallel (phases of
 * ceil(fft/hop) interleaved block sets). */
void mfo_ref_conv_ola_f32(const float* x, int64_t nx, const float* h, int K, int fft,
                          float* y, int nthreads) {
    int64_t ny = nx + K - 1;
    int hop = fft - K + 1;
    int64_t nblocks = (nx + hop - 1) / hop;
    c32* hk = (c32*)calloc((size_t)fft, sizeof(c32));
    c32* H = (c32*)malloc(sizeof(c32) * (size_t)fft);
    for (int i = 0; i < K; ++i) hk[i].x = h[i];
    mfo_ref_fft_c64((const float*)hk, (float*)H, fft, 1, 0, 1);
    memset(y, 0, sizeof(float) * (size_t)ny);
    int phases = (fft + hop - 1) / hop;
    int nt = mfo_set_threads(nthreads);
    for (int ph = 0; ph < phases; ++ph) {
#pragma omp parallel num_threads(nt)
        {
            c32* blk = (c32*)malloc(sizeof(c32) * (size_t)fft);
            c32* S = (c32*)malloc(sizeof(c32) * (size_t)fft);
            c32* R = (c32*)malloc(sizeof(c32) * (size_t)fft);
#pragma omp for schedule(static)
            for (int64_t bi = ph; bi < nblocks; bi += phases) {
                int64_t pos = bi * hop;
                int64_t chunk = nx - pos < hop ? nx - pos : hop;
                for (int i = 0; i < fft; ++i) {
                    blk[i].x = i < chunk ? x[pos + i] : 0.0f;
                    blk[i].y = 0.0f;
                }
                mfo_ref_fft_c64((const float*)blk, (float*)S, fft, 1, 0, 1);
                for (int i = 0; i < fft; ++i) S[i] = cmul32(S[i], H[i]);
                mfo_ref_fft_c64((const float*)S, (float*)R, fft, 1, 1, 1);
                for (int i = 0; i < fft; ++i) {
                    int64_t o = pos + i;
                    if (o < ny) y[o] += R[i].x;
                }
            }
            free(blk);
            free(S);
            free(R);
        }
    }
    free(hk);
    free(H);
}

/* FP64 linear convolution y = x * h via FP64 FFT overlap-add (same block
 * arithmetic as above, FP64 throughout).  Ground truth for the convolver. */
void mfo_conv_f64(const double* x, int64_t nx, const double* h, int K, int fft, double* y,
                  int nthreads) {
    int64_t ny = nx + K - 1;
    int hop = fft - K + 1;
    int64_t nblocks = (nx + hop - 1) / hop;
    double* hk = (double*)calloc((size_t)fft * 2, sizeof(double));
    double* H = (double*)malloc(sizeof(double) * 2 * (size_t)fft);
    for (int i = 0; i < K; ++i) hk[2 * i] = h[i];
    mfo_fft_c128(hk, H, fft, 1, -1, 1);
    memset(y, 0, sizeof(double) * (size_t)ny);
    int phases = (fft + hop - 1) / hop;
    int nt = mfo_set_threads(nthreads);
    for (int ph = 0; ph < phases; ++ph) {
#pragma omp parallel num_threads(nt)
        {
            double* blk = (double*)malloc(sizeof(double) * 2 * (size_t)fft);
            double* S = (double*)malloc(sizeof(double) * 2 * (size_t)fft);
#pragma omp for schedule(static)
            for (int64_t bi = ph; bi < nblocks; bi += phases) {
                int64_t pos = bi * hop;
                int64_t chunk = nx - pos < hop ? nx - pos : hop;
                for (int i = 0; i < fft; ++i) {
                    blk[2 * i] = i < chunk ? x[pos + i] : 0.0;
                    blk[2 * i + 1] = 0.0;
                }
                mfo_fft_c128(blk, S, fft, 1, -1, 1);
                for (int i = 0; i < fft; ++i) {
                    double sr = S[2 * i], si = S[2 * i + 1], hr = H[2 * i], hi = H[2 * i + 1];
                    S[2 * i] = sr * hr - si * hi;
                    S[2 * i + 1] = sr * hi + si * hr;
                }
                mfo_fft_c128(S, blk, fft, 1, +1, 1);
                for (int i = 0; i < fft; ++i) {
                    int64_t o = pos + i;
                    if (o < ny) y[o] += blk[2 * i] / (double)fft;
                }
            }
            free(blk);
            free(S);
        }
    }
    free(hk);
    free(H);
}

/* FP64 adjoint of y = x * h for L = 0.5*||y - t||^2 given g = dL/dy (length
 * nx + K - 1):  dx[n] = sum_k g[n+k] h[k]  (length nx),
 *               dh[k] = sum_n g[n+k] x[n]  (length K).
 * Computed as correlations via FP64 FFTs of length >= nx + K - 1 (one shot,
 * no blocking: exact up to FP64 rounding). */
void mfo_conv_adjoint_f64(const double* x, int64_t nx, const double* h, int K,
                          const double* g, double* dx, double* dh) {
    int64_t ny = nx + K - 1;
    int64_t L = 1;
    while (L < ny) L <<= 1;
    double* G = (double*)calloc((size_t)L * 2, sizeof(double));
    double* A = (double*)calloc((size_t)L * 2, sizeof(double));
    for (int64_t i = 0; i < ny; ++i) G[2 * i] = g[i];
    mfo_fft_c128(G, G, L, 1, -1, 0);
    /* dx = corr(g, h): DX = G * conj(FFT(h)) */
    for (int i = 0; i < K; ++i) A[2 * i] = h[i];
    mfo_fft_c128(A, A, L, 1, -1, 0);
    for (int64_t i = 0; i < L; ++i) {
        double gr = G[2 * i], gi = G[2 * i + 1], ar = A[2 * i], ai = -A[2 * i + 1];
        A[2 * i] = gr * ar - gi * ai;
        A[2 * i + 1] = gr * ai + gi * ar;
    }
    mfo_fft_c128(A, A, L, 1, +1, 0);
    for (int64_t i = 0; i < nx; ++i) dx[i] = A[2 * i] / (double)L;
    /* dh = corr(g, x) */
    memset(A, 0, sizeof(double) * 2 * (size_t)L);
    for (int64_t i = 0; i < nx; ++i) A[2 * i] = x[i];
    mfo_fft_c128(A, A, L, 1, -1, 0);
    for (int64_t i = 0; i < L; ++i) {
        double gr = G[2 * i], gi = G[2 * i + 1], ar = A[2 * i], ai = -A[2 * i + 1];
        A[2 * i] = gr * ar - gi * ai;
        A[2 * i + 1] = gr * ai + gi * ar;
    }
    mfo_fft_c128(A, A, L, 1, +1, 0);
    for (int k = 0; k < K; ++k) dh[k] = A[2 * k] / (double)L;
    free(G);
    free(A);
}

/* Circular cross-correlation R[m] = Re IFFT(FFT(a) conj(FFT(b))) with a, b
 * zero-padded or truncated to fft (Correlate.swift:31-61), FP64. */
void mfo_corr_f64(const double* a, int64_t na, const double* b, int64_t nb, int fft,
                  double* r) {
    double* A = (double*)calloc((size_t)fft * 2, sizeof(double));
    double* B = (double*)calloc((size_t)fft * 2, sizeof(double));
    for (int64_t i = 0; i < na && i < fft; ++i) A[2 * i] = a[i];
    for (int64_t i = 0; i < nb && i < fft; ++i) B[2 * i] = b[i];
    mfo_fft_c128(A, A, fft, 1, -1, 1);
    mfo_fft_c128(B, B, fft, 1, -1, 1);
    for (int i = 0; i < fft; ++i) {
        double ar = A[2 * i], ai = A[2 * i + 1], br = B[2 * i], bi = B[2 * i + 1];
        A[2 * i] = ar * br + ai * bi;
        A[2 * i + 1] = ai * br - ar * bi;
    }
    mfo_fft_c128(A, A, fft, 1, +1, 1);
    for (int i = 0; i < fft; ++i) r[i] = A[2 * i] / (double)fft;
    free(A);
    free(B);
}

/* FP32 restatement of Correlator.cross (Correlate.swift:31-48). */
void mfo_ref_corr_f32(const float* a, int64_t na, const float* b, int64_t nb, int fft,
                      float* r) {
    c32* A = (c32*)calloc((size_t)fft, sizeof(c32));
    c32* B = (c32*)calloc((size_t)fft, sizeof(c32));
    c32* FA = (c32*)malloc(sizeof(c32) * (size_t)fft);
    c32* FB = (c32*)malloc(sizeof(c32) * (size_t)fft);
    for (int64_t i = 0; i < na && i < fft; ++i) A[i].x = a[i];
    for (int64_t i = 0; i < nb && i < fft; ++i) B[i].x = b[i];
    mfo_ref_fft_c64((const float*)A, (float*)FA, fft, 1, 0, 1);
    mfo_ref_fft_c64((const float*)B, (float*)FB, fft, 1, 0, 1);
    for (int i = 0; i < fft; ++i) {
        c32 p = {FA[i].x * FB[i].x + FA[i].y * FB[i].y, FA[i].y * FB[i].x - FA[i].x * FB[i].y};
        A[i] = p;
    }
    mfo_ref_fft_c64((const float*)A, (float*)FA, fft, 1, 1, 1);
    for (int i = 0; i < fft; ++i) r[i] = FA[i].x;
    free(A);
    free(B);
    free(FA);
    free(FB);
}

/* ------------------------------------------------------------------------ */
/* Windows (Sources/MetalFFT/DSP/Window.swift:32-95), FP64                   */
/* ------------------------------------------------------------------------ */

static double bessel_i0(double x) {
    /* power series, as Window.swift:98-108 */
    double result = 1.0, term = 1.0, hx = x / 2.0;
    for (int k = 1; k <= 30; ++k) {
        term *= (hx * hx) / (double)(k * k);
        result += term;
        if (term < 1e-12 * result) break;
    }
    return result;
}

/* kind: 0 hann (vDSP_HANN_NORM), 1 hamming, 2 blackman, 3 flat-top,
 *       4 kaiser(beta), 5 rectangular.
 * vDSP definitions (Apple vDSP reference, full window, denominator N):
 *   hann NORM: 0.8165 * (1 - cos(2*pi*n/N))
 *   hamming:   0.54 - 0.46 * cos(2*pi*n/N)
 *   blackman:  0.42 - 0.5 * cos(2*pi*n/N) + 0.08 * cos(4*pi*n/N)
 * flat-top and kaiser follow Window.swift:51-75. */
void mfo_window(int kind, int n, double beta, double* w) {
    for (int k = 0; k < n; ++k) {
        double x = 2.0 * MFO_PI * (double)k / (double)n;
        switch (kind) {
            case 0: w[k] = 0.8165 * (1.0 - cos(x)); break;
            case 1: w[k] = 0.54 - 0.46 * cos(x); break;
            case 2: w[k] = 0.42 - 0.5 * cos(x) + 0.08 * cos(2.0 * x); break;
            case 3: {
                double a0 = 0.21557895, a1 = 0.41663158, a2 = 0.277263158, a3 = 0.083578947,
                       a4 = 0.006947368;
                w[k] = a0 - a1 * cos(x) + a2 * cos(2.0 * x) - a3 * cos(3.0 * x) + a4 * cos(4.0 * x);
                break;
            }
            case 4: {
                double halfN = (double)(n - 1) / 2.0;
                double t = ((double)k - halfN) / halfN;
                double v = 1.0 - t * t;
                w[k] = bessel_i0(beta * sqrt(v > 0.0 ? v : 0.0)) / bessel_i0(beta);
                break;
            }
            default: w[k] = 1.0; break;
        }
    }
}

/* ---- STFT / Welch PSD / coherence (FP64) ---------------------------------
 * STFT.analyze (Sources/MetalFFT/DSP/STFT.swift:79-88, frame() :97-107):
 * frames at pos = 0, hop, 2 hop, ... while pos + fft <= n; frame f = FFT of
 * w[i] * x[f*hop + i] with zero imaginary part, all fft bins.
 * PSD.welch (DSP/PSD.swift:18-58): sum over frames of |X|^2 per bin, times
 * 1 / (frames * sum(w^2) * sample_rate).
 * PSD.coherence (DSP/PSD.swift:71-134): Sxx, Syy, Sxy = sum |A|^2, |B|^2,
 * A conj(B) over the frames of min(na, nb) samples; C = |Sxy|^2 / (Sxx Syy),
 * 0 where the denominator is not positive. */

int64_t mfo_stft_frames(int64_t n, int fft, int hop) {
    if (n < fft || hop <= 0) return 0;
    return (n - fft) / hop + 1;
}

/* out: frames x fft complex128 */
void mfo_stft(const double* x, int64_t n, int fft, int hop, const double* w, double* out) {
    const int64_t frames = mfo_stft_frames(n, fft, hop);
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < frames; ++f) {
        double* z = out + 2 * f * fft;
        for (int i = 0; i < fft; ++i) {
            z[2 * i] = w[i] * x[f * hop + i];
            z[2 * i + 1] = 0.0;
        }
        mfo_fft_c128(z, z, fft, 1, -1, 1);
    }
}

/* returns the frame count; out: fft values */
int64_t mfo_welch(const double* x, int64_t n, int fft, int hop, const double* w, double sample_rate, double* out) {
    const int64_t frames = mfo_stft_frames(n, fft, hop);
    memset(out, 0, sizeof(double) * fft);
    if (frames == 0) return 0;
    double* spec = (double*)malloc(sizeof(double) * 2 * frames * fft);
    mfo_stft(x, n, fft, hop, w, spec);
    double wss = 0.0;
    for (int i = 0; i < fft; ++i) wss += w[i] * w[i];
    for (int64_t f = 0; f < frames; ++f)
        for (int k = 0; k < fft; ++k) {
            const double* z = spec + 2 * (f * fft + k);
            out[k] += z[0] * z[0] + z[1] * z[1];
        }
    const double inv = 1.0 / ((double)frames * wss * sample_rate);
    for (int k = 0; k < fft; ++k) out[k] *= inv;
    free(spec);
    return frames;
}

int64_t mfo_coherence(const double* a, int64_t na, const double* b, int64_t nb, int fft, int hop, const double* w,
                      double* out) {
    const int64_t n = na < nb ? na : nb;
    const int64_t frames = mfo_stft_frames(n, fft, hop);
    memset(out, 0, sizeof(double) * fft);
    if (frames == 0) return 0;
    double* sa = (double*)malloc(sizeof(double) * 2 * frames * fft);
    double* sb = (double*)malloc(sizeof(double) * 2 * frames * fft);
    mfo_stft(a, n, fft, hop, w, sa);
    mfo_stft(b, n, fft, hop, w, sb);
    for (int k = 0; k < fft; ++k) {
        double sxx = 0, syy = 0, xr = 0, xi = 0;
        for (int64_t f = 0; f < frames; ++f) {
            const double* p = sa + 2 * (f * fft + k);
            const double* q = sb + 2 * (f * fft + k);
            sxx += p[0] * p[0] + p[1] * p[1];
            syy += q[0] * q[0] + q[1] * q[1];
            xr += p[0] * q[0] + p[1] * q[1];
            xi += p[1] * q[0] - p[0] * q[1];
        }
        const double den = sxx * syy;
        out[k] = den > 0.0 ? (xr * xr + xi * xi) / den : 0.0;
    }
    free(sa);
    free(sb);
    return frames;
}

/* ---- PSD.crossSpectral (FP64) ----------------------------------------------
 * Sources/MetalFFT/DSP/CrossSpectral.swift:56-152 with the per-bin kernel
 * Resources/fft_cross_spectral.metal:29-63: every frame (pos + fft <= n,
 * pos += hop) of each channel is windowed and transformed; per frame and bin
 * the kernel forms p_c = |X_c|^2, S_ij = X_i conj(X_j) for the upper-triangle
 * pairs (0,1), (0,2), ..., (C-2,C-1) and the per-frame coherence
 * |S_ij|^2 / max(p_i p_j, 1e-30); the host sums the three over frames and
 * divides by the frame count (CrossSpectral.swift:134-151).  No frames: all
 * zeros.  x: channels x n; power: channels x fft; cross: pairs x fft
 * complex128; coh: pairs x fft.  Returns the frame count. */
int64_t mfo_cross_spectral(const double* x, int channels, int64_t n, int fft, int hop, const double* w,
                           double* power, double* cross, double* coh) {
    const int pairs = channels * (channels - 1) / 2;
    const int64_t frames = mfo_stft_frames(n, fft, hop);
    memset(power, 0, sizeof(double) * channels * fft);
    if (pairs) {
        memset(cross, 0, sizeof(double) * 2 * pairs * fft);
        memset(coh, 0, sizeof(double) * pairs * fft);
    }
    if (frames == 0) return 0;
    double* spec = (double*)malloc(sizeof(double) * 2 * frames * fft * channels);
    for (int c = 0; c < channels; ++c) mfo_stft(x + c * n, n, fft, hop, w, spec + 2 * (int64_t)c * frames * fft);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < fft; ++k) {
        for (int64_t f = 0; f < frames; ++f) {
            int pr = 0;
            for (int i = 0; i < channels; ++i) {
                const double* u = spec + 2 * (((int64_t)i * frames + f) * fft + k);
                const double pi = u[0] * u[0] + u[1] * u[1];
                power[i * fft + k] += pi;
                for (int j = i + 1; j < channels; ++j, ++pr) {
                    const double* v = spec + 2 * (((int64_t)j * frames + f) * fft + k);
                    const double pj = v[0] * v[0] + v[1] * v[1];
                    const double sr = u[0] * v[0] + u[1] * v[1];
                    const double si = u[1] * v[0] - u[0] * v[1];
                    cross[2 * (pr * fft + k)] += sr;
                    cross[2 * (pr * fft + k) + 1] += si;
                    const double den = pi * pj > 1e-30 ? pi * pj : 1e-30;
                    coh[pr * fft + k] += (sr * sr + si * si) / den;
                }
            }
        }
        const double inv = 1.0 / (double)frames;
        for (int c = 0; c < channels; ++c) power[c * fft + k] *= inv;
        for (int q = 0; q < pairs; ++q) {
            cross[2 * (q * fft + k)] *= inv;
            cross[2 * (q * fft + k) + 1] *= inv;
            coh[q * fft + k] *= inv;
        }
    }
    free(spec);
    return frames;
}
