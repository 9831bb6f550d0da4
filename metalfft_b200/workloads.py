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
