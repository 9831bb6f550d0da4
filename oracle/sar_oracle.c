/*
 * sar_oracle.c -- FP64 oracle of the SAR range-Doppler chain.  TEST
 * INFRASTRUCTURE ONLY (see oracle.c).
 *
 * Restates:
 *   SARSimulator.simulate          src/radar/sar_simulator.swift:93-159
 *     (chirp exp(j*pi*Kr*dt^2), two-way phase exp(-j*4*pi*R/lambda), window
 *      |dt| <= Tp/2), plus a per-target reflection phase;
 *   addNoise                       sar_simulator.swift:161-204 (complex
 *     Gaussian noise, std per component sqrt(P/2/10^(snr/10)), P = mean
 *     power of the non-zero samples), drawn here from a counter-based
 *     generator (splitmix64 finaliser) so the device simulator is comparable;
 *   generateChirpReference         sar_simulator.swift:209-224;
 *   range compression              src/fft_sar_fused.metal:246-293 with
 *     H = conj(FFT(chirp)) (src/radar/rda_fused_pipeline.swift:189-196),
 *     IFFT scaled by 1/N;
 *   azimuth FFT                    rda_fused_pipeline.swift:224-242 (unscaled
 *     forward FFT along the pulse index for every range bin);
 * and, with no reference counterpart, the per-pulse phase e^{j phi_p}, the
 * sharpness loss L = sum |I|^4 and its analytic gradient dL/dphi;
 *   RCMC + azimuth matched filter  src/radar/rda_kernels.metal:103-240 with
 *     the reference's signs or the focusing ones (mfo_sar_focus below).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SAR_C 299792458.0
#define SAR_PI 3.14159265358979323846

void mfo_fft_c128(const double* in, double* out, int64_t n, int64_t batch, int sign, int nthreads);

typedef struct {
    int64_t pulses, range_n, chirp_samples;
    double bandwidth, sample_rate, prf, velocity, carrier, center_range;
} mfo_sar_params;

typedef struct {
    double range_m, azimuth_m, amplitude, phase;
} mfo_sar_target;

static uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double unit_open(uint64_t seed, uint64_t idx) {
    return ((double)(mix64(seed ^ mix64(idx)) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

/* raw: pulses x range_n complex128, pulse-major */
void mfo_sar_simulate(const mfo_sar_params* p, const mfo_sar_target* tg, int nt, double snr_db, uint64_t seed,
                      double* raw) {
    const int64_t na = p->pulses, nr = p->range_n;
    const double tp = (double)p->chirp_samples / p->sample_rate;
    const double kr = p->bandwidth / tp;
    const double lambda = SAR_C / p->carrier;
    const double tau0 = 2.0 * p->center_range / SAR_C - (double)(nr / 2) / p->sample_rate;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < na; ++q) {
        const double eta = (double)(q - na / 2) / p->prf;
        for (int64_t r = 0; r < nr; ++r) {
            const double tr = tau0 + (double)r / p->sample_rate;
            double re = 0.0, im = 0.0;
            for (int i = 0; i < nt; ++i) {
                const double dx = p->velocity * eta - tg[i].azimuth_m;
                const double R = sqrt(tg[i].range_m * tg[i].range_m + dx * dx);
                const double dt = tr - 2.0 * R / SAR_C;
                if (fabs(dt) <= tp / 2.0) {
                    const double ph = SAR_PI * kr * dt * dt - 4.0 * SAR_PI * R / lambda + tg[i].phase;
                    re += tg[i].amplitude * cos(ph);
                    im += tg[i].amplitude * sin(ph);
                }
            }
            /* the device stores the signal in FP32 before adding noise */
            raw[2 * (q * nr + r)] = (double)(float)re;
            raw[2 * (q * nr + r) + 1] = (double)(float)im;
        }
    }
    double s = 0.0, c = 0.0;
    for (int64_t i = 0; i < na * nr; ++i) {
        const double m = raw[2 * i] * raw[2 * i] + raw[2 * i + 1] * raw[2 * i + 1];
        if (m > 0.0) {
            s += m;
            c += 1.0;
        }
    }
    if (c <= 0.0) return;
    const double sigma = sqrt((s / c) / pow(10.0, snr_db / 10.0) / 2.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < na * nr; ++i) {
        const double u1 = unit_open(seed, 2 * (uint64_t)i), u2 = unit_open(seed, 2 * (uint64_t)i + 1);
        const double rr = sigma * sqrt(-2.0 * log(u1));
        raw[2 * i] += rr * cos(2.0 * SAR_PI * u2);
        raw[2 * i + 1] += rr * sin(2.0 * SAR_PI * u2);
    }
}

/* image[k][r] (pulses x range_n complex128) of raw * e^{j phi_p} */
void mfo_sar_image(const mfo_sar_params* p, const double* raw, const double* chirp, const double* phi,
                   double* image, double* rc_out) {
    const int64_t na = p->pulses, nr = p->range_n;
    double* H = (double*)malloc(sizeof(double) * 2 * nr);
    mfo_fft_c128(chirp, H, nr, 1, -1, 1);
    double* rc = rc_out ? rc_out : (double*)malloc(sizeof(double) * 2 * na * nr);
    double* X = (double*)malloc(sizeof(double) * 2 * na * nr);
    mfo_fft_c128(raw, X, nr, na, -1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < na; ++q)
        for (int64_t k = 0; k < nr; ++k) {
            double* z = X + 2 * (q * nr + k);
            const double hr = H[2 * k], hi = -H[2 * k + 1];
            const double zr = z[0] * hr - z[1] * hi, zi = z[0] * hi + z[1] * hr;
            z[0] = zr;
            z[1] = zi;
        }
    mfo_fft_c128(X, rc, nr, na, +1, 0);
    const double inv = 1.0 / (double)nr;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < na; ++q) {
        const double c = cos(phi[q]), s = sin(phi[q]);
        for (int64_t r = 0; r < nr; ++r) {
            double* z = rc + 2 * (q * nr + r);
            const double a = z[0] * inv, b = z[1] * inv;
            z[0] = a * c - b * s;
            z[1] = a * s + b * c;
        }
    }
    /* azimuth FFT: transpose to range-major lines, FFT, transpose back */
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nr; ++r)
        for (int64_t q = 0; q < na; ++q) {
            X[2 * (r * na + q)] = rc[2 * (q * nr + r)];
            X[2 * (r * na + q) + 1] = rc[2 * (q * nr + r) + 1];
        }
    mfo_fft_c128(X, X, na, nr, -1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nr; ++r)
        for (int64_t k = 0; k < na; ++k) {
            image[2 * (k * nr + r)] = X[2 * (r * na + k)];
            image[2 * (k * nr + r) + 1] = X[2 * (r * na + k) + 1];
        }
    free(H);
    free(X);
    if (!rc_out) free(rc);
}

/* L = sum |I|^4 and dL/dphi_p = -sum_r Im(u_p[r] conj(B[p][r])),
 * B[p][r] = sum_k 4 |I[k][r]|^2 I[k][r] e^{+2 pi i p k / na} */
double mfo_sar_loss_grad(const mfo_sar_params* p, const double* raw, const double* chirp, const double* phi,
                         double* dphi) {
    const int64_t na = p->pulses, nr = p->range_n;
    double* I = (double*)malloc(sizeof(double) * 2 * na * nr);
    double* u = (double*)malloc(sizeof(double) * 2 * na * nr);
    mfo_sar_image(p, raw, chirp, phi, I, u);
    double L = 0.0;
    double* G = (double*)malloc(sizeof(double) * 2 * na * nr);
    for (int64_t r = 0; r < nr; ++r)
        for (int64_t k = 0; k < na; ++k) {
            const double a = I[2 * (k * nr + r)], b = I[2 * (k * nr + r) + 1];
            const double m = a * a + b * b;
            L += m * m;
            G[2 * (r * na + k)] = 4.0 * m * a;
            G[2 * (r * na + k) + 1] = 4.0 * m * b;
        }
    mfo_fft_c128(G, G, na, nr, +1, 0); /* B, range-major */
    for (int64_t q = 0; q < na; ++q) {
        double s = 0.0;
        for (int64_t r = 0; r < nr; ++r) {
            const double ur = u[2 * (q * nr + r)], ui = u[2 * (q * nr + r) + 1];
            const double br = G[2 * (r * na + q)], bi = G[2 * (r * na + q) + 1];
            /* Im(u conj(B)) = ui*br - ur*bi */
            s -= ui * br - ur * bi;
        }
        dphi[q] = s;
    }
    free(I);
    free(u);
    free(G);
    return L;
}

/* Focusing of the range-Doppler image (FP64): RCMC and the azimuth matched
 * filter of the reference's RDA (src/radar/rda_kernels.metal:103-240,
 * rda_fused_pipeline.swift:248-368), then the azimuth inverse FFT (1/na).
 * Per Doppler row k (FFT order: f_a = k/na * prf below na/2, (k-na)/na * prf
 * above): ratio = lambda f_a / (2 v); valid when |ratio| < 0.95;
 * q = sqrt(1 - ratio^2); dR = R0 (1/q - 1) (0 when not valid), R0 = center
 * range; shift = dR / rho, rho = c / (2 fs).  RCMC output r = sum over taps
 * j = -3..4 of in[c0 + r + j] * sinc(frac - j) * (0.54 - 0.46 cos(2 pi (j+3)/7)),
 * src = r + d, d = -shift (reference) or +shift, c0 = floor(d), frac = d - c0.
 * Filter: phase = 4 pi q R0(r) / lambda, R0(r) = R0 + (r - nr/2) rho;
 * H = exp(-j phase) (reference) or exp(+j phase); 0 when not valid.
 * rd and out: na x nr complex128, Doppler / azimuth major. */
void mfo_sar_focus(const mfo_sar_params* p, const double* rd, int reference_signs, double* out) {
    const int64_t na = p->pulses, nr = p->range_n;
    const double lambda = SAR_C / p->carrier, rho = SAR_C / (2.0 * p->sample_rate);
    double* tmp = (double*)malloc(sizeof(double) * 2 * na * nr);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < na; ++k) {
        const double fa = (double)(k < na / 2 ? k : k - na) / (double)na * p->prf;
        const double ratio = lambda * fa / (2.0 * p->velocity);
        const int valid = fabs(ratio) < 0.95;
        const double q = valid ? sqrt(1.0 - ratio * ratio) : 1.0;
        const double shift = valid ? p->center_range * (1.0 / q - 1.0) / rho : 0.0;
        const double d = reference_signs ? -shift : shift;
        const double c0 = floor(d), frac = d - c0;
        double w[8];
        for (int j = -3; j <= 4; ++j) {
            const double x = frac - (double)j;
            const double sv = fabs(x) < 1e-6 ? 1.0 : sin(SAR_PI * x) / (SAR_PI * x);
            w[j + 3] = sv * (0.54 - 0.46 * cos(2.0 * SAR_PI * (double)(j + 3) / 7.0));
        }
        for (int64_t r = 0; r < nr; ++r) {
            double ar = 0.0, ai = 0.0;
            for (int j = -3; j <= 4; ++j) {
                const int64_t idx = (int64_t)c0 + r + j;
                if (idx < 0 || idx >= nr) continue;
                ar += rd[2 * (k * nr + idx)] * w[j + 3];
                ai += rd[2 * (k * nr + idx) + 1] * w[j + 3];
            }
            double hr = 0.0, hi = 0.0;
            if (valid) {
                const double ph = 4.0 * SAR_PI * q * (p->center_range + (double)(r - nr / 2) * rho) / lambda;
                hr = cos(ph);
                hi = reference_signs ? -sin(ph) : sin(ph);
            }
            tmp[2 * (k * nr + r)] = ar * hr - ai * hi;
            tmp[2 * (k * nr + r) + 1] = ar * hi + ai * hr;
        }
    }
    /* inverse FFT along azimuth for every range column, 1/na */
    double* col = (double*)malloc(sizeof(double) * 2 * na * nr);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nr; ++r)
        for (int64_t k = 0; k < na; ++k) {
            col[2 * (r * na + k)] = tmp[2 * (k * nr + r)];
            col[2 * (r * na + k) + 1] = tmp[2 * (k * nr + r) + 1];
        }
    mfo_fft_c128(col, col, na, nr, +1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nr; ++r)
        for (int64_t k = 0; k < na; ++k) {
            out[2 * (k * nr + r)] = col[2 * (r * na + k)] / (double)na;
            out[2 * (k * nr + r) + 1] = col[2 * (r * na + k) + 1] / (double)na;
        }
    free(tmp);
    free(col);
}
