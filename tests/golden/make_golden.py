"""Generates tests/golden/*.npz: seeded inputs and their FP64 transforms.

The reference ships no golden vectors (its tests draw unseeded
Float.random), so the fixtures are produced here by the FP64 oracle and
accepted only if numpy's pocketfft (the stand-in for the reference's vDSP
comparison path) agrees to 1e-13.  Run from the repository root:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    fx = {}
    for n, seed in [(64, 101), (512, 102), (4096, 103)]:
        x = O.uniform_c64((2, n), seed=seed)
        X = O.truth(x)
        np.testing.assert_allclose(X, np.fft.fft(x.astype(np.complex128), axis=-1), rtol=0, atol=1e-11)
        fx["x_%d" % n] = x
        fx["X_%d" % n] = X
    np.savez_compressed(os.path.join(HERE, "fft_golden.npz"), **fx)

    rng = np.random.default_rng(104)
    x = rng.standard_normal(1000).astype(np.float32)
    h = (rng.standard_normal(63) * np.exp(-np.arange(63) / 20.0)).astype(np.float32)
    y = O.conv64(x, h, 128)
    np.testing.assert_allclose(y, np.convolve(x.astype(np.float64), h.astype(np.float64)), atol=1e-11)
    t = rng.standard_normal(len(y)).astype(np.float32)
    dx, dh = O.conv_adjoint64(x, h, y - t)
    np.savez_compressed(os.path.join(HERE, "conv_golden.npz"), x=x, h=h, y=y, t=t, dx=dx, dh=dh,
                        fft=np.int64(128))
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
