// sar.cu -- SAR range-Doppler chain with FP16 storage and its phase adjoint.
//
// Reference: RDAFusedPipeline (src/radar/rda_fused_pipeline.swift:131-242):
// fused range compression per pulse (FFT -> * conj(FFT(chirp)) -> IFFT,
// src/fft_sar_fused.metal:246-293, N_FFT = 4096 hard-coded), then the azimuth
// FFT as transpose_2d -> batched FFT -> transpose_2d, each step its own
// command buffer with FP32 device data; FP16 only in threadgroup memory
// (fft_sar_fused_fp16.metal:10-33).  The simulator is SARSimulator
// (src/radar/sar_simulator.swift:79-245).
//
// Here (two passes over HBM, FP16 storage with power-of-two block scales):
//   pass A  k_sar_range   one pulse per CTA: FP16 samples * pulse scale *
//                         e^{j phi_p} -> FFT -> * H -> IFFT -> FP16 with a new
//                         per-pulse scale, pulse-major (the scale of each
//                         pulse travels with it through the corner turn)
//   pass B  k_sar_azimuth a tile of C range columns x all pulses per CTA: the
//                         corner turn is the tile load itself (each row of the
//                         tile is C consecutive range bins); FFT along azimuth
//                         -> FP16 image (azimuth-major, one scale per range
//                         column) and/or the adjoint of L = sum |I|^4 with
//                         respect to phi: G = 4|I|^2 I, B = sum_k G W^{-pk}
//                         (one more FFT on the registers), per-tile partials
//                         of dphi_p = -sum_r Im(u_p[r] conj(B[p][r]))
//   reduce  k_sar_reduce  partials summed over tiles in a fixed order (FP64)
// The range-compressed intermediate between the passes is FP16 with per-pulse
// scales by default; mfft_sar_set_intermediate switches it to FP32 (no
// scales), which the phase adjoint needs to meet FP64 gradients to ~1e-5.
#include <cuda_fp16.h>

#include <vector>

#include "capi_internal.h"
#include "stockham.cuh"

namespace mfft {
namespace {

constexpr double C_LIGHT = 299792458.0;
constexpr double PI_D = 3.14159265358979323846;
constexpr int SAR_E = 16;

struct SarGeom {
    long long na, nr;
    double fs, prf, v, tp, kr, lambda, tau0;
};

SarGeom make_geom(const mfft_sar_params& p) {
    SarGeom g;
    g.na = p.pulses;
    g.nr = p.range_n;
    g.fs = p.sample_rate;
    g.prf = p.prf;
    g.v = p.velocity;
    g.tp = (double)p.chirp_samples / p.sample_rate;
    g.kr = p.bandwidth / g.tp;
    g.lambda = C_LIGHT / p.carrier;
    g.tau0 = 2.0 * p.center_range / C_LIGHT - (double)(p.range_n / 2) / p.sample_rate;
    return g;
}

// counter-based generator (splitmix64 finaliser), identical on host and device
__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ inline double unit_open(uint64_t seed, uint64_t idx) {
    return ((double)(mix64(seed ^ mix64(idx)) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// A CTA covers SIG_T consecutive range samples of one pulse (blockIdx.x =
// pulse * chunks + chunk).  The slant range R of each target depends on the
// pulse only: the CTA forms R, 2R/c and 4 pi R / lambda once per target (in
// shared memory, SIG_T targets at a time) and every sample reads them, with
// the same FP64 expressions as a per-sample evaluation.
constexpr int SIG_T = 256;
__global__ void __launch_bounds__(SIG_T)
    k_sar_signal(float2* __restrict__ raw, SarGeom g, const mfft_sar_target* __restrict__ tg, int nt) {
    __shared__ double s_delay[SIG_T], s_rph[SIG_T], s_ph[SIG_T], s_amp[SIG_T];
    const long long chunks = (g.nr + SIG_T - 1) / SIG_T;
    const long long p = blockIdx.x / chunks, r = (blockIdx.x % chunks) * SIG_T + threadIdx.x;
    const double eta = (double)(p - g.na / 2) / g.prf;
    const double tr = g.tau0 + (double)r / g.fs;
    double re = 0.0, im = 0.0;
    for (int i0 = 0; i0 < nt; i0 += SIG_T) {
        const int i = i0 + threadIdx.x;
        if (i < nt) {
            const double dx = g.v * eta - tg[i].azimuth_m;
            const double R = sqrt(tg[i].range_m * tg[i].range_m + dx * dx);
            s_delay[threadIdx.x] = 2.0 * R / C_LIGHT;
            s_rph[threadIdx.x] = 4.0 * PI_D * R / g.lambda;
            s_ph[threadIdx.x] = tg[i].phase;
            s_amp[threadIdx.x] = tg[i].amplitude;
        }
        __syncthreads();
        const int n = nt - i0 < SIG_T ? nt - i0 : SIG_T;
        for (int j = 0; j < n; ++j) {
            const double dt = tr - s_delay[j];
            if (fabs(dt) <= g.tp / 2.0) {
                const double ph = PI_D * g.kr * dt * dt - s_rph[j] + s_ph[j];
                double sn, cs;
                sincos(ph, &sn, &cs);
                re += s_amp[j] * cs;
                im += s_amp[j] * sn;
            }
        }
        __syncthreads();
    }
    if (r < g.nr) raw[p * g.nr + r] = make_float2((float)re, (float)im);
}

// per-block partial sums of |s|^2 over non-zero samples and their count
__global__ void k_sar_power(const float2* __restrict__ raw, long long n, double* __restrict__ part) {
    __shared__ double ss[256], sc[256];
    double s = 0.0, c = 0.0;
    for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
        const float2 v = raw[i];
        const double m = (double)v.x * v.x + (double)v.y * v.y;
        if (m > 0.0) {
            s += m;
            c += 1.0;
        }
    }
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            ss[threadIdx.x] += ss[threadIdx.x + o];
            sc[threadIdx.x] += sc[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = ss[0];
        part[2 * blockIdx.x + 1] = sc[0];
    }
}

// the noise standard deviation per component, once: the partial sums added in
// block order (FP64), sqrt(P / (2 * 10^(snr/10))) with P the mean |s|^2 of the
// non-zero samples; -1 when every sample is zero (no noise is added)
__global__ void k_sar_sigma(double* __restrict__ part, int nparts, double snr_db) {
    if (threadIdx.x != 0) return;
    double s = 0.0, c = 0.0;
    for (int i = 0; i < nparts; ++i) {
        s += part[2 * i];
        c += part[2 * i + 1];
    }
    part[2 * nparts] = c <= 0.0 ? -1.0 : sqrt((s / c) / pow(10.0, snr_db / 10.0) / 2.0);
}

// complex Gaussian noise: per-sample Box-Muller on two counter-based uniforms,
// std per component *sigma_p (k_sar_sigma)
__global__ void k_sar_noise(float2* __restrict__ raw, long long n, const double* __restrict__ sigma_p, uint64_t seed) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const double sigma = *sigma_p;
    if (sigma < 0.0) return;
    const double u1 = unit_open(seed, 2 * (uint64_t)idx), u2 = unit_open(seed, 2 * (uint64_t)idx + 1);
    const double rr = sigma * sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    const float2 v = raw[idx];
    raw[idx] = make_float2((float)(v.x + rr * cs), (float)(v.y + rr * sn));
}

// power-of-two block scale s with max|v| / s < 2^15 (1 for an all-zero block)
__device__ __forceinline__ float block_scale(float mx) {
    if (!(mx > 0.f)) return 1.f;
    int e;
    frexpf(mx, &e);
    return ldexpf(1.f, e - 15);
}

__device__ __forceinline__ float cta_max(float v, float* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    float m = red[0];
    for (int i = 1; i < nw; ++i) m = fmaxf(m, red[i]);
    return m;
}

__global__ void k_sar_quantize(const float2* __restrict__ raw, long long nr, __half2* __restrict__ out,
                               float* __restrict__ scale) {
    __shared__ float red[32];
    const long long p = blockIdx.x;
    const float2* row = raw + p * nr;
    float mx = 0.f;
    for (long long i = threadIdx.x; i < nr; i += blockDim.x) {
        const float2 v = row[i];
        mx = fmaxf(mx, fmaxf(fabsf(v.x), fabsf(v.y)));
    }
    const float s = block_scale(cta_max(mx, red));
    const float inv = 1.f / s;
    for (long long i = threadIdx.x; i < nr; i += blockDim.x) {
        const float2 v = row[i];
        out[p * nr + i] = __floats2half2_rn(v.x * inv, v.y * inv);
    }
    if (threadIdx.x == 0) scale[p] = s;
}

// the range-compressed intermediate: FP16 (times a per-pulse scale) or FP32
__device__ __forceinline__ float2 ld_rc(const __half2* p) { return __half22float2(*p); }
__device__ __forceinline__ float2 ld_rc(const float2* p) { return *p; }

// pass A: range compression of one pulse per CTA; RC = __half2 (FP16 with a
// per-pulse scale) or float2 (FP32, scale 1).  Up to NR = 8192 two CTAs share
// an SM (64 registers a thread at 512 threads, without spills; 2 x 70 KB of
// shared memory): twice the warps to hide the exchanges' latency.
template <int NR>
constexpr int range_min_blocks() { return NR <= 8192 ? 2 : 1; }
template <int NR, class RC>
__global__ void __launch_bounds__(NR / SAR_E, range_min_blocks<NR>()) k_sar_range(const __half2* __restrict__ raw, const float* __restrict__ pscale,
                                                           const float* __restrict__ phase, const float2* __restrict__ H,
                                                           const float2* __restrict__ tw, RC* __restrict__ rc,
                                                           float* __restrict__ rc_scale) {
    constexpr int T = NR / SAR_E;
    extern __shared__ __align__(16) float2 smem[];
    __shared__ float red[32];
    const long long p = blockIdx.x;
    const int t = threadIdx.x;
    float sp, cp;
    sincosf(phase[p], &sp, &cp);
    const float sc = pscale[p];
    const float2 rot = make_float2(cp * sc, sp * sc);
    const __half2* rawp = raw + p * NR + t;  // this thread's samples t + m*T of pulse p
    float2 v[SAR_E];
#pragma unroll
    for (int m = 0; m < SAR_E; ++m) v[m] = cmul(__half22float2(rawp[m * T]), rot);
    // forward transform, times conj(H), inverse transform through one call site
    // (two inlined transforms get interleaved and need more registers)
#pragma unroll 1
    for (int ph = 0; ph < 2; ++ph) {
        fft_regs<NR, SAR_E, (T <= 32)>(v, t, PadLineS{smem}, tw);
        if (ph == 0) {
#pragma unroll
            for (int m = 0; m < SAR_E; ++m) v[m] = cconj(cmul(v[m], __ldg(H + t + m * T)));
        }
    }
    float mx = 0.f;
    const float inv_n = 1.f / (float)NR;
#pragma unroll
    for (int m = 0; m < SAR_E; ++m) {
        v[m] = make_float2(v[m].x * inv_n, -v[m].y * inv_n);
        mx = fmaxf(mx, fmaxf(fabsf(v[m].x), fabsf(v[m].y)));
    }
    RC* rcp = rc + p * NR + t;
    if constexpr (sizeof(RC) == sizeof(float2)) {
#pragma unroll
        for (int m = 0; m < SAR_E; ++m) rcp[m * T] = v[m];
        if (t == 0) rc_scale[p] = 1.f;
    } else {
        const float s = block_scale(cta_max(mx, red));
        const float inv = 1.f / s;
#pragma unroll
        for (int m = 0; m < SAR_E; ++m) rcp[m * T] = __floats2half2_rn(v[m].x * inv, v[m].y * inv);
        if (t == 0) rc_scale[p] = s;
    }
}

template <int NA>
struct AzGeom {
    static constexpr int T = NA / SAR_E;
    static constexpr int C = (16384 / NA) < 16 ? (16384 / NA) : 16;  // range columns per CTA
    static constexpr int THREADS = T * C;
};

// pass B: azimuth FFT of C range columns; IMAGE: write the FP16 image;
// GRAD: per-tile partials of dL/dphi and of L = sum |I|^4
template <int NA, bool IMAGE, bool GRAD, bool INV = false, class RC = __half2>
__global__ void __launch_bounds__(AzGeom<NA>::THREADS)
    k_sar_azimuth(const RC* __restrict__ rc, const float* __restrict__ rc_scale, long long nr,
                  const float2* __restrict__ tw, __half2* __restrict__ image, float* __restrict__ image_scale,
                  float* __restrict__ dphi_part, double* __restrict__ loss_part) {
    constexpr int T = AzGeom<NA>::T, C = AzGeom<NA>::C;
    extern __shared__ __align__(16) float2 smem[];
    __shared__ float red[32][C];
    __shared__ double lred[32];
    const long long tile = blockIdx.x;
    const int c = threadIdx.x % C, t = threadIdx.x / C;
    const long long col = tile * C + c;
    // rows t + m*T of column col: a base pointer and a stride of T rows
    const RC* rcol = rc + (long long)t * nr + col;
    const long long rstep = (long long)T * nr;
    float2 v[SAR_E];
#pragma unroll
    for (int m = 0; m < SAR_E; ++m) {
        const int p = t + m * T;
        const float2 u = ld_rc(rcol + m * rstep);
        const float s = __ldg(rc_scale + p);
        v[m] = make_float2(u.x * s, INV ? -u.y * s : u.y * s);
    }
    // the azimuth transform and, for the gradient, the transform of conj(G)
    // through one call site (two inlined transforms get interleaved and need
    // more registers)
#pragma unroll 1
    for (int ph = 0; ph < (GRAD ? 2 : 1); ++ph) {
        fft_regs<NA, SAR_E, false>(v, t, ColPadLine<C>{smem, c}, tw);  // ph 0: v[m] = I[k = t + m*T][col]
        if (ph == 1) break;                                          // ph 1: v[m] = conj(B[p]), p = t + m*T
        if constexpr (INV) {
            // inverse transform along azimuth: conj(FFT(conj(x))) / NA
            const float sc = 1.0f / (float)NA;
#pragma unroll
            for (int m = 0; m < SAR_E; ++m) v[m] = make_float2(v[m].x * sc, -v[m].y * sc);
        }
        if constexpr (IMAGE) {
            float mx = 0.f;
#pragma unroll
            for (int m = 0; m < SAR_E; ++m) mx = fmaxf(mx, fmaxf(fabsf(v[m].x), fabsf(v[m].y)));
            // max over the T threads of column c: lanes differing in t share a warp
            // when C < 32 (t varies across lane bits above log2 C)
#pragma unroll
            for (int o = 16; o >= C; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            const int w = threadIdx.x >> 5;
            if ((threadIdx.x & 31) < C) red[w][c] = mx;
            __syncthreads();
            float cm = 0.f;
            for (int i = 0; i < (AzGeom<NA>::THREADS + 31) / 32; ++i) cm = fmaxf(cm, red[i][c]);
            const float s = block_scale(cm);
            const float inv = 1.f / s;
            __half2* icol = image + (long long)t * nr + col;
#pragma unroll
            for (int m = 0; m < SAR_E; ++m) icol[m * rstep] = __floats2half2_rn(v[m].x * inv, v[m].y * inv);
            if (t == 0) image_scale[col] = s;
        }
        if constexpr (GRAD) {
            double lsum = 0.0;
#pragma unroll
            for (int m = 0; m < SAR_E; ++m) {
                const float a2 = v[m].x * v[m].x + v[m].y * v[m].y;
                lsum += (double)a2 * (double)a2;
                v[m] = make_float2(4.f * a2 * v[m].x, -4.f * a2 * v[m].y);  // conj(G)
            }
            // the warp's part of the loss waits in shared memory, not in registers,
            // while conj(G) is transformed
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
            if ((threadIdx.x & 31) == 0) lred[threadIdx.x >> 5] = lsum;
        }
    }
    if constexpr (GRAD) {
        // per pulse p = t + m*T: -Im(u conj(B)) with v = conj(B), i.e. -Im(u v),
        // summed over the C columns of the tile (c is the low part of the lane id)
        // and stored as soon as it is formed
#pragma unroll
        for (int m = 0; m < SAR_E; ++m) {
            const int p = t + m * T;
            const float2 u0 = ld_rc(rcol + m * rstep);
            const float s = __ldg(rc_scale + p);
            const float2 u = make_float2(u0.x * s, u0.y * s);
            float d = -(u.x * v[m].y + u.y * v[m].x);
#pragma unroll
            for (int o = 1; o < C && o < 32; o <<= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
            if (c == 0) dphi_part[tile * NA + p] = d;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int i = 0; i < (AzGeom<NA>::THREADS + 31) / 32; ++i) tot += lred[i];
            loss_part[tile] = tot;
        }
    }
}

// dphi[p] = sum over tiles (fixed order); loss = sum of the tile losses
// dphi[p] = sum over tiles of part[tile][p], loss = sum of loss_part: FP64 in a
// fixed order.  CTA b < ceil(na / 32) owns pulses 32b .. 32b + 31 (lane = pulse,
// so a warp reads 128 contiguous bytes of a tile); its 32 warps sum contiguous
// runs of tiles in tile order, then lane l adds the 32 runs in warp order.  The
// last CTA sums the loss partials: contiguous runs per thread, then a fixed
// pairwise tree.
constexpr int SAR_RED_THREADS = 1024;
__global__ void __launch_bounds__(SAR_RED_THREADS)
    k_sar_reduce(const float* __restrict__ part, long long tiles, long long na, float* __restrict__ dphi,
                 const double* __restrict__ loss_part, double* __restrict__ loss) {
    __shared__ double red[SAR_RED_THREADS];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const long long pulse_ctas = (na + 31) / 32;
    if (blockIdx.x < pulse_ctas) {
        const long long p = (long long)blockIdx.x * 32 + l;
        const long long run = (tiles + 31) / 32, i0 = w * run, i1 = i0 + run < tiles ? i0 + run : tiles;
        double s = 0.0;
        if (p < na)
            for (long long i = i0; i < i1; ++i) s += part[i * na + p];
        red[threadIdx.x] = s;
        __syncthreads();
        if (w == 0 && p < na) {
            double t = 0.0;
            for (int q = 0; q < 32; ++q) t += red[q * 32 + l];
            dphi[p] = (float)t;
        }
    } else if (loss) {
        const long long run = (tiles + SAR_RED_THREADS - 1) / SAR_RED_THREADS, i0 = threadIdx.x * run;
        const long long i1 = i0 + run < tiles ? i0 + run : tiles;
        double s = 0.0;
        for (long long i = i0; i < i1; ++i) s += loss_part[i];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int h = SAR_RED_THREADS / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) *loss = red[0];
    }
}

// Per Doppler row: RCMC taps and the azimuth matched filter's phase (cycles
// alpha + beta * r), computed on the host in FP64.
struct RcmcRow {
    double alpha, beta;  // filter phase in cycles for range bin r
    float w[8];          // interpolation taps j = -3 .. 4
    int c0;              // input index of tap j for output r: r + c0 + j
    int valid;           // |lambda f_a / 2v| < 0.95 (else the row is zero)
    float sign;          // +1: exp(+j phase); -1: exp(-j phase)
    int pad;
};

// focus pass 1: one Doppler row per CTA.  In: the range-Doppler image (FP16,
// one scale per range column); out: RCMC'd and matched-filtered row (FP16,
// one scale per row), the input layout of the inverse azimuth pass.
template <int NR>
__global__ void __launch_bounds__(NR / SAR_E) k_sar_rcmc(const __half2* __restrict__ rd, const float* __restrict__ rd_scale,
                                                          const RcmcRow* __restrict__ rows, __half2* __restrict__ out,
                                                          float* __restrict__ out_scale) {
    constexpr int T = NR / SAR_E;
    extern __shared__ __align__(16) float2 line[];
    __shared__ float red[32];
    const long long k = blockIdx.x;
    const int t = threadIdx.x;
#pragma unroll
    for (int m = 0; m < SAR_E; ++m) {
        const int r = t + m * T;
        const float2 u = __half22float2(rd[k * NR + r]);
        const float sc = __ldg(rd_scale + r);
        line[r] = make_float2(u.x * sc, u.y * sc);
    }
    __syncthreads();
    const RcmcRow R = rows[k];
    // matched-filter phasors e^{+-j 2 pi (alpha + beta r)} of this thread's bins
    // r = t + m*T: the phase of r = t formed in FP64 and reduced to one cycle,
    // times products of at most three of e^{+-j 2 pi beta T {1, 2, 4, 8}}
    float2 h[SAR_E];
    {
        auto phasor = [&](double cyc) {
            const float f = (float)(cyc - floor(cyc));
            float sn, cs;
            sincospif(2.0f * f, &sn, &cs);
            return R.valid ? make_float2(cs, R.sign * sn) : make_float2(0.f, 0.f);
        };
        const float2 base = phasor(fma((double)t, R.beta, R.alpha));
        const double bt = R.beta * (double)T;
        const float2 s1 = phasor(bt), s2 = phasor(2.0 * bt), s4 = phasor(4.0 * bt), s8 = phasor(8.0 * bt);
        float2 u[4];
        u[0] = base;
        u[1] = cmul(base, s1);
        u[2] = cmul(base, s2);
        u[3] = cmul(u[1], s2);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float2 w4 = cmul(u[q], s4);
            h[q] = u[q];
            h[q + 4] = w4;
            h[q + 8] = cmul(u[q], s8);
            h[q + 12] = cmul(w4, s8);
        }
    }
    float2 v[SAR_E];
    float mx = 0.f;
#pragma unroll
    for (int m = 0; m < SAR_E; ++m) {
        const int r = t + m * T;
        const int lo = r + R.c0 - 3;  // taps lo .. lo + 7
        float2 acc = make_float2(0.f, 0.f);
        if (lo >= 0 && lo + 7 < NR) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float2 x = line[lo + j];
                acc.x = fmaf(x.x, R.w[j], acc.x);
                acc.y = fmaf(x.y, R.w[j], acc.y);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int idx = lo + j;
                if (idx >= 0 && idx < NR) {
                    const float2 x = line[idx];
                    acc.x = fmaf(x.x, R.w[j], acc.x);
                    acc.y = fmaf(x.y, R.w[j], acc.y);
                }
            }
        }
        v[m] = cmul(acc, h[m]);
        mx = fmaxf(mx, fmaxf(fabsf(v[m].x), fabsf(v[m].y)));
    }
    const float s = block_scale(cta_max(mx, red));
    const float inv = 1.f / s;
#pragma unroll
    for (int m = 0; m < SAR_E; ++m) out[k * NR + t + m * T] = __floats2half2_rn(v[m].x * inv, v[m].y * inv);
    if (t == 0) out_scale[k] = s;
}

typedef void (*rcmc_fn)(int grid, cudaStream_t, const __half2*, const float*, const RcmcRow*, __half2*, float*);
template <int NR>
void l_rcmc(int grid, cudaStream_t s, const __half2* rd, const float* rds, const RcmcRow* rows, __half2* out,
            float* outs) {
    k_sar_rcmc<NR><<<grid, NR / SAR_E, NR * 8, s>>>(rd, rds, rows, out, outs);
}

template <class RC>
using range_fn_t = void (*)(int grid, cudaStream_t, const __half2*, const float*, const float*, const float2*,
                            const float2*, RC*, float*);
template <class RC>
using az_fn_t = void (*)(int grid, cudaStream_t, const RC*, const float*, long long, const float2*, __half2*, float*,
                         float*, double*);
typedef az_fn_t<__half2> az_fn;

template <int NR, class RC>
void l_range(int grid, cudaStream_t s, const __half2* raw, const float* ps, const float* ph, const float2* H,
             const float2* tw, RC* rc, float* rcs) {
    k_sar_range<NR, RC><<<grid, NR / SAR_E, spad_size(NR) * 8, s>>>(raw, ps, ph, H, tw, rc, rcs);
}
template <int NA, bool IMAGE, bool GRAD, bool INV = false, class RC = __half2>
void l_az(int grid, cudaStream_t s, const RC* rc, const float* rcs, long long nr, const float2* tw, __half2* img,
          float* imgs, float* dp, double* lp) {
    k_sar_azimuth<NA, IMAGE, GRAD, INV, RC><<<grid, AzGeom<NA>::THREADS, spad_size(NA) * AzGeom<NA>::C * 8, s>>>(
        rc, rcs, nr, tw, img, imgs, dp, lp);
}
template <int NR>
cudaError_t prep_range() {
    const int sm = spad_size(NR) * 8;
    cudaError_t e = cudaFuncSetAttribute(k_sar_range<NR, __half2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_sar_range<NR, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    // the largest shared-memory carveout, so that range_min_blocks CTAs fit on an SM
    e = cudaFuncSetAttribute(k_sar_range<NR, __half2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_sar_range<NR, float2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_sar_rcmc<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, NR * 8);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_sar_rcmc<NR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
}
template <int NA, bool IMAGE, bool GRAD, bool INV, class RC>
cudaError_t prep_az1() {
    return cudaFuncSetAttribute(k_sar_azimuth<NA, IMAGE, GRAD, INV, RC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                spad_size(NA) * AzGeom<NA>::C * 8);
}
template <int NA>
cudaError_t prep_az() {
    cudaError_t e;
    if ((e = prep_az1<NA, true, false, false, __half2>())) return e;
    if ((e = prep_az1<NA, false, true, false, __half2>())) return e;
    if ((e = prep_az1<NA, true, false, true, __half2>())) return e;
    if ((e = prep_az1<NA, true, true, false, __half2>())) return e;
    if ((e = prep_az1<NA, true, false, false, float2>())) return e;
    if ((e = prep_az1<NA, false, true, false, float2>())) return e;
    return prep_az1<NA, true, true, false, float2>();
}

struct RangeK {
    int n;
    range_fn_t<__half2> f;
    range_fn_t<float2> f32;
    cudaError_t (*prep)();
    rcmc_fn rcmc;
};
struct AzK {
    int n, cols;
    az_fn fwd, bwd, both, inv;
    az_fn_t<float2> fwd32, bwd32, both32;
    cudaError_t (*prep)();
};
#define MFFT_RANGE(N) {N, &l_range<N, __half2>, &l_range<N, float2>, &prep_range<N>, &l_rcmc<N>}
const RangeK g_range[] = {MFFT_RANGE(512),  MFFT_RANGE(1024), MFFT_RANGE(2048),
                          MFFT_RANGE(4096), MFFT_RANGE(8192), MFFT_RANGE(16384)};
#define MFFT_AZ(N)                                                                                              \
    {N, AzGeom<N>::C, &l_az<N, true, false>, &l_az<N, false, true>, &l_az<N, true, true>, &l_az<N, true, false, true>, \
     &l_az<N, true, false, false, float2>, &l_az<N, false, true, false, float2>, &l_az<N, true, true, false, float2>, \
     &prep_az<N>}
const AzK g_az[] = {MFFT_AZ(64), MFFT_AZ(128), MFFT_AZ(256), MFFT_AZ(512), MFFT_AZ(1024), MFFT_AZ(2048), MFFT_AZ(4096)};

const BatchedKernel* e16(int n) {
    int cnt = 0;
    const BatchedKernel* ks = batched_kernels(&cnt);
    for (int i = 0; i < cnt; ++i)
        if (ks[i].n == n && ks[i].e == 16) return &ks[i];
    return nullptr;
}

}  // namespace
}  // namespace mfft

using namespace mfft;

struct mfft_sar {
    mfft_ctx* ctx = nullptr;
    mfft_sar_params prm{};
    const RangeK* rk = nullptr;
    const AzK* ak = nullptr;
    float2* tw_r = nullptr;
    float2* tw_a = nullptr;
    float2* H = nullptr;
    __half2* rc = nullptr;  // range-compressed pulses, FP16 pulse-major
    float2* rc32 = nullptr; // the same in FP32 (allocated when selected)
    int rc_fp32 = 0;        // MFFT_SAR_RC_FP16 / MFFT_SAR_RC_FP32
    float* rc_scale = nullptr;
    float* dphi_part = nullptr;
    double* loss_part = nullptr;
    long long tiles = 0;
    cudaGraphExec_t graph = nullptr;
    const void* g_key[9] = {};
    // focusing (allocated by the first mfft_sar_focus)
    __half2* rd2 = nullptr;      // RCMC'd, matched-filtered rows, FP16
    float* rd2_scale = nullptr;  // one scale per Doppler row
    RcmcRow* rows[2] = {};       // per-row taps / filter: [0] focusing signs, [1] reference signs
};

static int check_params(const mfft_sar_params* p) {
    if (!p) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "params is NULL");
    if (!is_pow2_in(p->pulses, 64, 4096))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, p->pulses, -1, -1, "pulses must be a power of two 64..4096, got %lld",
                         (long long)p->pulses);
    if (!is_pow2_in(p->range_n, 512, 16384))
        return set_error(MFFT_ERR_UNSUPPORTED_SIZE, p->range_n, -1, -1,
                         "range_n must be a power of two 512..16384, got %lld", (long long)p->range_n);
    if (p->chirp_samples < 1 || p->chirp_samples > p->range_n || !(p->sample_rate > 0) || !(p->prf > 0) ||
        !(p->bandwidth > 0) || !(p->carrier > 0))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "invalid SAR parameters");
    return MFFT_SUCCESS;
}

extern "C" int mfft_sar_default_params(int64_t pulses, int64_t range_n, int64_t chirp_samples, double tbp,
                                       mfft_sar_params* out) {
    if (!out || chirp_samples < 1 || !(tbp > 0)) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "bad arguments");
    out->pulses = pulses;
    out->range_n = range_n;
    out->chirp_samples = chirp_samples;
    out->bandwidth = 100e6;
    out->sample_rate = (double)chirp_samples * out->bandwidth / tbp;  // Tp*fs = samples, B*Tp = tbp
    out->prf = 1000.0;
    out->velocity = 100.0;
    out->carrier = 10e9;
    out->center_range = 20000.0;
    return check_params(out);
}

extern "C" int mfft_sar_chirp_reference(const mfft_sar_params* p, void* chirp) {
    int st = check_params(p);
    if (st) return st;
    if (!chirp) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "chirp is NULL");
    const SarGeom g = make_geom(*p);
    float2* out = (float2*)chirp;
    for (int64_t i = 0; i < p->range_n; ++i) out[i] = make_float2(0.f, 0.f);
    const int64_t ns = p->chirp_samples, half = ns / 2;
    for (int64_t i = 0; i < ns; ++i) {
        const double t = (double)(i - half) / p->sample_rate;
        const double ph = PI_D * g.kr * t * t;
        const int64_t idx = i < half ? p->range_n - half + i : i - half;
        if (idx < p->range_n) out[idx] = make_float2((float)cos(ph), (float)sin(ph));
    }
    return MFFT_SUCCESS;
}

extern "C" int mfft_sar_simulate(mfft_ctx* ctx, const mfft_sar_params* p, const mfft_sar_target* targets,
                                 int ntargets, double snr_db, uint64_t seed, void* raw, void* stream) {
    int st = check_params(p);
    if (st) return st;
    if (!raw || ntargets < 0 || (ntargets > 0 && !targets))
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "bad simulator arguments");
    if (!ctx) {
        st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    DeviceGuard gd(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    const SarGeom g = make_geom(*p);
    const long long n = g.na * g.nr;
    mfft_sar_target* dt = nullptr;
    double* part = nullptr;
    const int nparts = 1024;
    cudaError_t e = cudaMallocAsync(&dt, sizeof(mfft_sar_target) * (ntargets > 0 ? ntargets : 1), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&part, sizeof(double) * (2 * nparts + 1), s);
    if (e != cudaSuccess) return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "simulator buffers: %s", cudaGetErrorString(e));
    if (ntargets > 0) e = cudaMemcpyAsync(dt, targets, sizeof(mfft_sar_target) * ntargets, cudaMemcpyHostToDevice, s);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    k_sar_signal<<<(unsigned)(g.na * ((g.nr + SIG_T - 1) / SIG_T)), SIG_T, 0, s>>>((float2*)raw, g, dt, ntargets);
    k_sar_power<<<nparts, 256, 0, s>>>((const float2*)raw, n, part);
    k_sar_sigma<<<1, 32, 0, s>>>(part, nparts, snr_db);
    k_sar_noise<<<blocks, 256, 0, s>>>((float2*)raw, n, part + 2 * nparts, seed);
    cudaFreeAsync(dt, s);
    cudaFreeAsync(part, s);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "SAR simulator");
    return MFFT_SUCCESS;
}

extern "C" int mfft_sar_quantize(mfft_ctx* ctx, int64_t pulses, int64_t range_n, const void* raw, void* raw_h,
                                 float* pulse_scale, void* stream) {
    if (!raw || !raw_h || !pulse_scale || pulses < 1 || range_n < 1)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "bad quantize arguments");
    if (!ctx) {
        int st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    DeviceGuard gd(ctx->device);
    k_sar_quantize<<<(unsigned)pulses, 256, 0, (cudaStream_t)stream>>>((const float2*)raw, range_n, (__half2*)raw_h,
                                                                       pulse_scale);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "SAR quantize");
    return MFFT_SUCCESS;
}

extern "C" int mfft_sar_destroy(mfft_sar* s) {
    if (!s) return MFFT_SUCCESS;
    DeviceGuard gd(s->ctx->device);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    cudaFree(s->H);
    cudaFree(s->rc);
    cudaFree(s->rc32);
    cudaFree(s->rc_scale);
    cudaFree(s->dphi_part);
    cudaFree(s->loss_part);
    cudaFree(s->rd2);
    cudaFree(s->rd2_scale);
    cudaFree(s->rows[0]);
    cudaFree(s->rows[1]);
    delete s;
    return MFFT_SUCCESS;
}

extern "C" int mfft_sar_create(mfft_ctx* ctx, const mfft_sar_params* p, const void* chirp_ref, mfft_sar** out) {
    if (!out) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "out is NULL");
    *out = nullptr;
    int st = check_params(p);
    if (st) return st;
    if (!chirp_ref) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "chirp_ref is NULL");
    if (!ctx) {
        st = mfft_context_shared(&ctx);
        if (st) return st;
    }
    DeviceGuard gd(ctx->device);
    mfft_sar* s = new mfft_sar();
    s->ctx = ctx;
    s->prm = *p;
    for (const auto& k : g_range)
        if (k.n == p->range_n) s->rk = &k;
    for (const auto& k : g_az)
        if (k.n == p->pulses) s->ak = &k;
    s->tiles = p->range_n / s->ak->cols;
    BatchedBinding br, ba;
    st = bind_batched(ctx, e16((int)p->range_n), &br);
    if (!st) st = bind_batched(ctx, e16((int)p->pulses), &ba);
    s->tw_r = br.tw;
    s->tw_a = ba.tw;
    cudaError_t e = cudaSuccess;
    if (!st) {
        e = s->rk->prep();
        if (e == cudaSuccess) e = s->ak->prep();
        if (e != cudaSuccess) st = cuda_error(e, "SAR kernel attributes");
    }
    const long long na = p->pulses, nr = p->range_n;
    if (!st) {
        e = cudaMalloc(&s->H, sizeof(float2) * nr * 2);
        if (e == cudaSuccess) e = cudaMalloc(&s->rc, sizeof(__half2) * na * nr);
        if (e == cudaSuccess) e = cudaMalloc(&s->rc_scale, sizeof(float) * na);
        if (e == cudaSuccess) e = cudaMalloc(&s->dphi_part, sizeof(float) * s->tiles * na);
        if (e == cudaSuccess) e = cudaMalloc(&s->loss_part, sizeof(double) * s->tiles);
        if (e != cudaSuccess) st = set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "SAR buffers: %s", cudaGetErrorString(e));
    }
    if (!st) {
        // H = conj(FFT(chirp_ref)): conj(FFT(c)) computed as the inverse-scaled
        // transform of conj(c) would change the scale, so transform and conjugate
        std::vector<float2> h((size_t)nr);
        memcpy(h.data(), chirp_ref, sizeof(float2) * nr);
        float2* tmp = s->H + nr;
        e = cudaMemcpyAsync(tmp, h.data(), sizeof(float2) * nr, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = br.k->fwd(tmp, s->H, 1, br.tw, ctx->dev_err, ctx->stream, 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), s->H, sizeof(float2) * nr, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        for (auto& v : h) v.y = -v.y;
        if (e == cudaSuccess) e = cudaMemcpy(s->H, h.data(), sizeof(float2) * nr, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = cuda_error(e, "range matched filter");
    }
    if (st) {
        mfft_sar_destroy(s);
        return st;
    }
    *out = s;
    return MFFT_SUCCESS;
}

static int sar_pass_a(mfft_sar* s, const void* raw_h, const float* ps, const float* ph, cudaStream_t st) {
    if (s->rc_fp32)
        s->rk->f32((int)s->prm.pulses, st, (const __half2*)raw_h, ps, ph, s->H, s->tw_r, s->rc32, s->rc_scale);
    else
        s->rk->f((int)s->prm.pulses, st, (const __half2*)raw_h, ps, ph, s->H, s->tw_r, s->rc, s->rc_scale);
    return MFFT_SUCCESS;
}

// pass B in the selected intermediate precision: which = 0 image, 1 adjoint, 2 both
static void sar_pass_b(mfft_sar* s, int which, cudaStream_t st, void* image_h, float* image_scale) {
    const long long nr = s->prm.range_n;
    const int tiles = (int)s->tiles;
    if (s->rc_fp32) {
        const az_fn_t<float2> f = which == 0 ? s->ak->fwd32 : which == 1 ? s->ak->bwd32 : s->ak->both32;
        f(tiles, st, s->rc32, s->rc_scale, nr, s->tw_a, (__half2*)image_h, image_scale, s->dphi_part, s->loss_part);
    } else {
        const az_fn f = which == 0 ? s->ak->fwd : which == 1 ? s->ak->bwd : s->ak->both;
        f(tiles, st, s->rc, s->rc_scale, nr, s->tw_a, (__half2*)image_h, image_scale, s->dphi_part, s->loss_part);
    }
}

extern "C" int mfft_sar_set_intermediate(mfft_sar* s, int precision) {
    if (!s) return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "sar is NULL");
    if (precision != MFFT_SAR_RC_FP16 && precision != MFFT_SAR_RC_FP32)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, precision, -1, "unknown SAR intermediate precision %d",
                         precision);
    if (precision == MFFT_SAR_RC_FP32 && !s->rc32) {
        DeviceGuard gd(s->ctx->device);
        cudaError_t e = cudaMalloc(&s->rc32, sizeof(float2) * (size_t)s->prm.pulses * (size_t)s->prm.range_n);
        if (e != cudaSuccess) {
            s->rc32 = nullptr;
            return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "SAR FP32 intermediate: %s", cudaGetErrorString(e));
        }
    }
    s->rc_fp32 = precision == MFFT_SAR_RC_FP32;
    return MFFT_SUCCESS;
}

static int sar_check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? (int)MFFT_SUCCESS : cuda_error(e, what);
}

extern "C" int mfft_sar_forward(mfft_sar* s, const void* raw_h, const float* pulse_scale, const float* phase,
                                void* image_h, float* image_scale, void* stream) {
    if (!s || !raw_h || !pulse_scale || !phase || !image_h || !image_scale)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL argument");
    DeviceGuard gd(s->ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    sar_pass_a(s, raw_h, pulse_scale, phase, st);
    sar_pass_b(s, 0, st, image_h, image_scale);
    return sar_check_launch("SAR forward");
}

extern "C" int mfft_sar_backward_phase(mfft_sar* s, const void* raw_h, const float* pulse_scale, const float* phase,
                                       float* dphi, double* loss, void* stream) {
    if (!s || !raw_h || !pulse_scale || !phase || !dphi)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL argument");
    DeviceGuard gd(s->ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    sar_pass_a(s, raw_h, pulse_scale, phase, st);
    sar_pass_b(s, 1, st, nullptr, nullptr);
    k_sar_reduce<<<(unsigned)((s->prm.pulses + 31) / 32 + 1), SAR_RED_THREADS, 0, st>>>(
        s->dphi_part, s->tiles, s->prm.pulses, dphi, s->loss_part, loss);
    return sar_check_launch("SAR backward");
}

static void sar_enqueue_step(mfft_sar* s, const void* raw_h, const float* ps, const float* ph, void* image_h,
                             float* image_scale, float* dphi, double* loss, cudaStream_t st) {
    sar_pass_a(s, raw_h, ps, ph, st);
    sar_pass_b(s, 2, st, image_h, image_scale);
    k_sar_reduce<<<(unsigned)((s->prm.pulses + 31) / 32 + 1), SAR_RED_THREADS, 0, st>>>(
        s->dphi_part, s->tiles, s->prm.pulses, dphi, s->loss_part, loss);
}

extern "C" int mfft_sar_step_graph(mfft_sar* s, const void* raw_h, const float* pulse_scale, const float* phase,
                                   void* image_h, float* image_scale, float* dphi, double* loss, void* stream) {
    if (!s || !raw_h || !pulse_scale || !phase || !image_h || !image_scale || !dphi)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL argument");
    DeviceGuard gd(s->ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    const void* key[9] = {raw_h, pulse_scale, phase, image_h, image_scale, dphi, loss, stream,
                          s->rc_fp32 ? (const void*)s->rc32 : (const void*)s->rc};
    bool same = s->graph != nullptr;
    for (int i = 0; i < 9 && same; ++i) same = (key[i] == s->g_key[i]);
    if (!same) {
        if (s->graph) cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        // capture on a private stream, so a legacy default stream can be used too
        cudaStream_t cs;
        cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (e != cudaSuccess) return set_error(MFFT_ERR_NO_STREAM, -1, -1, -1, "capture stream: %s", cudaGetErrorString(e));
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            sar_enqueue_step(s, raw_h, pulse_scale, phase, image_h, image_scale, dphi, loss, cs);
            e = cudaStreamEndCapture(cs, &g);
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&s->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) {
            s->graph = nullptr;
            return cuda_error(e, "SAR graph capture");
        }
        for (int i = 0; i < 9; ++i) s->g_key[i] = key[i];
    }
    cudaError_t e = cudaGraphLaunch(s->graph, st);
    if (e != cudaSuccess) return cuda_error(e, "SAR graph launch");
    return MFFT_SUCCESS;
}

// Focusing of the range-Doppler image (rda_kernels.metal:103-240,
// rda_fused_pipeline.swift:248-368): per Doppler row f_a, RCMC by
// dR = R0 (1/sqrt(1 - (lambda f_a / 2v)^2) - 1) with an 8-tap Hamming-windowed
// sinc, times the azimuth matched filter of phase 4 pi q R0(r) / lambda, then
// the inverse azimuth FFT.  The reference reads its RCMC input at r - shift
// and multiplies by exp(-j phase); with its own echo model exp(-j 4 pi R /
// lambda) both move the target away from focus (in FP64: its RCMC lowers the
// peak below no correction at all, its filter moves the peak off the target),
// so the default here is r + shift and exp(+j phase); reference_signs = 1
// reproduces the reference's formulas exactly.  The reference takes PRF = 1000
// inside its RCMC kernel, which is its only PRF; the parameters' prf is used.
static void sar_rows(const mfft_sar_params& p, bool reference, std::vector<RcmcRow>& rows) {
    const long long na = p.pulses, nr = p.range_n;
    const double lambda = C_LIGHT / p.carrier, rho = C_LIGHT / (2.0 * p.sample_rate);
    rows.assign((size_t)na, RcmcRow{});
    for (long long k = 0; k < na; ++k) {
        RcmcRow& R = rows[(size_t)k];
        const double fa = (double)(k < na / 2 ? k : k - na) / (double)na * p.prf;
        const double ratio = lambda * fa / (2.0 * p.velocity);
        R.valid = fabs(ratio) < 0.95;
        const double q = R.valid ? sqrt(1.0 - ratio * ratio) : 1.0;
        const double shift = R.valid ? p.center_range * (1.0 / q - 1.0) / rho : 0.0;
        const double d = reference ? -shift : shift;
        const double c0 = floor(d), frac = d - c0;
        R.c0 = (int)c0;
        for (int j = -3; j <= 4; ++j) {
            const double x = frac - (double)j;
            const double sv = fabs(x) < 1e-6 ? 1.0 : sin(PI_D * x) / (PI_D * x);
            R.w[j + 3] = (float)(sv * (0.54 - 0.46 * cos(2.0 * PI_D * (double)(j + 3) / 7.0)));
        }
        // phase / (2 pi) = 2 q R0(r) / lambda, R0(r) = R0 + (r - nr/2) rho
        R.alpha = 2.0 * q * (p.center_range - (double)(nr / 2) * rho) / lambda;
        R.beta = 2.0 * q * rho / lambda;
        R.sign = reference ? -1.f : 1.f;
    }
}

extern "C" int mfft_sar_focus(mfft_sar* s, const void* rd_h, const float* rd_scale, void* focused_h,
                              float* focused_scale, int reference_signs, void* stream) {
    if (!s || !rd_h || !rd_scale || !focused_h || !focused_scale)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, -1, -1, "NULL argument");
    if (reference_signs != 0 && reference_signs != 1)
        return set_error(MFFT_ERR_INVALID_ARGUMENT, -1, reference_signs, -1, "reference_signs must be 0 or 1");
    DeviceGuard gd(s->ctx->device);
    const long long na = s->prm.pulses, nr = s->prm.range_n;
    cudaError_t e = cudaSuccess;
    if (!s->rd2) {
        e = cudaMalloc(&s->rd2, sizeof(__half2) * na * nr);
        if (e == cudaSuccess) e = cudaMalloc(&s->rd2_scale, sizeof(float) * na);
        if (e != cudaSuccess) {
            cudaFree(s->rd2);
            s->rd2 = nullptr;
            return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "SAR focus buffers: %s", cudaGetErrorString(e));
        }
    }
    RcmcRow*& rows = s->rows[reference_signs];
    if (!rows) {
        std::vector<RcmcRow> h;
        sar_rows(s->prm, reference_signs != 0, h);
        e = cudaMalloc(&rows, sizeof(RcmcRow) * na);
        if (e == cudaSuccess) e = cudaMemcpy(rows, h.data(), sizeof(RcmcRow) * na, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(rows);
            rows = nullptr;
            return set_error(MFFT_ERR_ALLOCATION, -1, -1, -1, "SAR focus rows: %s", cudaGetErrorString(e));
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    s->rk->rcmc((int)na, st, (const __half2*)rd_h, rd_scale, rows, s->rd2, s->rd2_scale);
    s->ak->inv((int)s->tiles, st, s->rd2, s->rd2_scale, nr, s->tw_a, (__half2*)focused_h, focused_scale, nullptr,
               nullptr);
    return sar_check_launch("SAR focus");
}
