"""Seeded synthetic workloads of the benchmark configurations (no datasets)."""
import numpy as np

MIXED_SIZES = [1 << k for k in range(6, 15)] + [1 << 20]
MIXED_MAX_POINTS = 1 << 26


def mixed_size_classes(seed=20261203, max_points=MIXED_MAX_POINTS, sizes=MIXED_SIZES):
    """Mixed-size batch: per-size counts ~ U{1..512} drawn in ascending size
    order from the seed, truncated so sum(count * n) <= max_points (the last
    drawn size is clamped to floor(remaining / n)).  Returns [(n, count)]."""
    rng = np.random.default_rng(seed)
    out, total = [], 0
    for n in sizes:
        c = int(rng.integers(1, 513))
        c = min(c, (max_points - total) // n)
        if c <= 0:
            break
        out.append((n, c))
        total += c * n
    return out


def normal_c64(n, seed):
    rng = np.random.default_rng(seed)
    z = rng.standard_normal(size=(int(n), 2), dtype=np.float32)
    return z.view(np.complex64)[:, 0]


def conv_workload(seed=20261203, nx=1 << 24, K=4095, decay=800.0):
    """Config 4: x ~ N(0,1) (nx), h[t] = n_t * exp(-t/decay) (K taps),
    target ~ N(0,1) of length nx + K - 1."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(nx, dtype=np.float32)
    h = (rng.standard_normal(K) * np.exp(-np.arange(K) / decay)).astype(np.float32)
    t = rng.standard_normal(nx + K - 1, dtype=np.float32)
    return x, h, t


def sar_targets(params, n=64, seed=20261203):
    """Config 5 scatterers: seeded range bins inside the chirp margin, seeded
    azimuth pulses in the middle three quarters, amplitude U[0.1, 1], phase
    U[0, 2 pi).  Returns a list of metalfft_b200.SARTarget."""
    from ._sar import SARTarget
    rng = np.random.default_rng(seed)
    c = 299792458.0
    out = []
    for _ in range(n):
        rb = int(rng.integers(params.chirp_samples, params.range_n - params.chirp_samples))
        pb = int(rng.integers(params.pulses // 8, 7 * params.pulses // 8))
        R0 = c * (params.tau0 + rb / params.sample_rate) / 2.0
        x = params.velocity * (pb - params.pulses / 2) / params.prf
        out.append(SARTarget(R0, x, float(rng.uniform(0.1, 1.0)), float(rng.uniform(0.0, 2 * np.pi))))
    return out


def sar_phase(pulses, seed=20261203, sigma=0.3):
    """Per-pulse phase-error vector ~ N(0, sigma) rad."""
    return np.random.default_rng(seed + 1).normal(0.0, sigma, pulses).astype(np.float32)
