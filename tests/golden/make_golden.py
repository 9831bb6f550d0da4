"""Generates tests/golden/*.npz: seeded inputs and their expected outputs,
computed WITHOUT the repository's oracle (oracle/), so that the tests can
check the oracle (and the CUDA path) against something that does not share
its code.

The reference ships no golden vectors (its XCTests draw unseeded
Float.random) and cannot run here (Swift + Metal + Accelerate), so the
expected outputs come from:
  - numpy's pocketfft in complex128 for every FFT (the stand-in for the
    reference's comparison path, Apple vDSP's vDSP_fft_zop);
  - numpy transliterations, line by line, of the reference's host loops:
      Convolver.init / apply      Sources/MetalFFT/DSP/Convolve.swift:19-76
      Correlator.cross / pack     Sources/MetalFFT/DSP/Correlate.swift:27-61
      FFTAnalyzer.analyze         Sources/MetalFFT/DSP/FFTAnalyzer.swift:93-116
      Window.flatTop / kaiser     Sources/MetalFFT/DSP/Window.swift:51-75,100-110
      MetalFFT.inverse            Sources/MetalFFT/FFT/MetalFFT.swift:56-65
    with the GPU transforms replaced by FP64 pocketfft;
  - np.convolve / np.correlate for the convolution adjoint (dL/dx, dL/dh of
    L = 0.5 ||y - t||^2, which has no reference counterpart).
The reference's edge cases are included: an empty signal, a signal shorter
than one hop, K = 1, a signal that ends on a hop boundary, correlator inputs
shorter and longer than fftSize.  Hann / Hamming / Blackman come from vDSP
(vDSP_hann_window with vDSP_HANN_NORM, vDSP_hamm_window, vDSP_blkman_window)
whose coefficients the reference does not spell out: they are not part of
these fixtures.

Run from the repository root:
    python tests/golden/make_golden.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


# ---- MetalFFT.forward / inverse with FP64 pocketfft ------------------------

def fft_forward(x):
    return np.fft.fft(np.asarray(x, np.complex128))


def fft_inverse(X):
    # MetalFFT.swift:56-65: conj(FFT(conj(X))) / N
    X = np.asarray(X, np.complex128)
    return np.conj(np.fft.fft(np.conj(X))) / len(X)


# ---- Convolver (Convolve.swift:19-76) --------------------------------------

class Convolver:
    def __init__(self, kernel, fft_size):
        assert fft_size > len(kernel)                      # :20-21 precondition
        self.block_size = fft_size                         # :22
        self.hop_size = fft_size - len(kernel) + 1         # :23
        self.kernel_len = len(kernel)                      # :24
        kc = np.zeros(fft_size, np.complex128)             # :27
        for i in range(len(kernel)):                       # :28-30
            kc[i] = complex(kernel[i], 0.0)
        self.kernel_spectrum = fft_forward(kc)             # :31

    def apply(self, signal):
        output_len = len(signal) + self.kernel_len - 1     # :37
        output = np.zeros(output_len, np.float64)          # :38
        block = np.zeros(self.block_size, np.complex128)   # :39
        pos = 0                                            # :43
        while pos < len(signal):                           # :44
            chunk = min(self.hop_size, len(signal) - pos)  # :45
            for i in range(chunk):                         # :48-50
                block[i] = complex(signal[pos + i], 0.0)
            for i in range(chunk, self.block_size):        # :51-53
                block[i] = 0.0
            s = fft_forward(block)                         # :55
            k = self.kernel_spectrum
            product = (s.real * k.real - s.imag * k.imag) + 1j * (s.real * k.imag + s.imag * k.real)  # :58-62
            r = fft_inverse(product)                       # :64
            for i in range(self.block_size):               # :67-70
                o = pos + i
                if o < output_len:
                    output[o] += r[i].real
            pos += self.hop_size                           # :72
        return output


def conv_adjoint(x, h, g):
    """y = x * h (full linear convolution): dL/dx[i] = sum_k g[i+k] h[k],
    dL/dh[k] = sum_i g[i+k] x[i]."""
    x = np.asarray(x, np.float64)
    h = np.asarray(h, np.float64)
    g = np.asarray(g, np.float64)
    dx = np.correlate(g, h, mode="valid")[: len(x)] if len(x) else np.zeros(0)
    dh = np.correlate(g, x, mode="valid")[: len(h)] if len(x) else np.zeros(len(h))
    return dx, dh


# ---- Correlator (Correlate.swift:27-61) ------------------------------------

def pack(samples, fft_size):
    buf = np.zeros(fft_size, np.complex128)                # :53-61
    n = min(len(samples), fft_size)
    for i in range(n):
        buf[i] = complex(samples[i], 0.0)
    return buf


def correlator_cross(a, b, fft_size):
    A = fft_forward(pack(a, fft_size))                     # :34-36
    B = fft_forward(pack(b, fft_size))                     # :35-37
    product = (A.real * B.real + A.imag * B.imag) + 1j * (A.imag * B.real - A.real * B.imag)  # :40-45
    return fft_inverse(product).real                       # :47-48


# ---- Window (Window.swift) and FFTAnalyzer (FFTAnalyzer.swift:93-116) ------

def flat_top(size):
    # Window.swift:51-63 (Float coefficients, written here in FP64)
    a0, a1, a2, a3, a4 = 0.21557895, 0.41663158, 0.277263158, 0.083578947, 0.006947368
    a0, a1, a2, a3, a4 = (float(np.float32(v)) for v in (a0, a1, a2, a3, a4))
    x = np.arange(size) / size
    return (a0 - a1 * np.cos(2 * np.pi * x) + a2 * np.cos(4 * np.pi * x) - a3 * np.cos(6 * np.pi * x)
            + a4 * np.cos(8 * np.pi * x))


def bessel_i0(x):
    # Window.swift:100-110
    result, term, half = 1.0, 1.0, x / 2.0
    for k in range(1, 31):
        term *= (half * half) / float(k * k)
        result += term
        if term < 1e-12 * result:
            break
    return result


def kaiser(size, beta):
    # Window.swift:66-73
    half_n = (size - 1) / 2.0
    i0b = bessel_i0(beta)
    return np.array([bessel_i0(beta * np.sqrt(max(0.0, 1.0 - ((k - half_n) / half_n) ** 2))) / i0b
                     for k in range(size)])


def analyze(samples, window, offset=0):
    size = len(window)
    assert offset + size <= len(samples)                   # :108 precondition
    w = np.asarray(window, np.float32)
    s = np.asarray(samples[offset:offset + size], np.float32)
    windowed = (s * w).astype(np.float32)                  # :109-111 vDSP_vmul (FP32)
    buf = windowed.astype(np.float64) + 0j                 # :112-114 pack
    return fft_forward(buf)                                # :115


def main():
    rng = np.random.default_rng(20261204)

    # FFT: MetalFFTTests.swift:25-35 inputs, U[-1,1) re and im
    fx = {}
    for n in [64, 512, 4096]:
        z = rng.uniform(-1, 1, size=(2, n, 2)).astype(np.float32)
        x = z.view(np.complex64)[..., 0]
        fx["x_%d" % n] = x
        fx["X_%d" % n] = np.fft.fft(x.astype(np.complex128), axis=-1)
        fx["Xi_%d" % n] = np.stack([fft_inverse(r) for r in x.astype(np.complex128)])
    np.savez_compressed(os.path.join(HERE, "fft_golden.npz"), **fx)

    # Convolver cases: (name, n, K, fftSize)
    conv = {}
    cases = [("main", 1000, 63, 128),      # several hops, ragged last block
             ("empty", 0, 33, 64),         # no block: K - 1 zeros
             ("short", 10, 63, 128),       # shorter than one hop
             ("k1", 300, 1, 64),           # hop = fftSize, identity-like
             ("boundary", 3 * 66, 63, 128),  # ends exactly on a hop boundary
             ("long_kernel", 700, 255, 256)]  # hop 2
    names = []
    for name, n, K, fft in cases:
        x = rng.standard_normal(n).astype(np.float32)
        h = (rng.standard_normal(K) * np.exp(-np.arange(K) / 20.0)).astype(np.float32)
        y = Convolver(h, fft).apply(x)
        assert len(y) == n + K - 1
        if n:
            assert np.max(np.abs(y - np.convolve(x.astype(np.float64), h.astype(np.float64)))) < 1e-10
        t = rng.standard_normal(len(y)).astype(np.float32)
        dx, dh = conv_adjoint(x, h, y - t)
        for k, v in dict(x=x, h=h, y=y, t=t, dx=dx, dh=dh, fft=np.int64(fft)).items():
            conv["%s_%s" % (name, k)] = v
        names.append(name)
    conv["cases"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "conv_golden.npz"), **conv)

    # Correlator cases: (name, na, nb, fftSize)
    corr = {}
    names = []
    for name, na, nb, fft in [("pad", 200, 150, 256),       # both zero-padded
                              ("trunc_b", 200, 300, 256),   # b longer than fftSize: truncated
                              ("trunc_both", 700, 900, 512),
                              ("empty_b", 64, 0, 128)]:
        a = rng.standard_normal(na).astype(np.float32)
        b = rng.standard_normal(nb).astype(np.float32)
        corr["%s_a" % name] = a
        corr["%s_b" % name] = b
        corr["%s_r" % name] = correlator_cross(a, b, fft)
        corr["%s_fft" % name] = np.int64(fft)
        names.append(name)
    a = rng.standard_normal(100).astype(np.float32)
    corr["auto_a"] = a
    corr["auto_b"] = a
    corr["auto_r"] = correlator_cross(a, a, 256)
    corr["auto_fft"] = np.int64(256)
    names.append("auto")
    corr["cases"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "corr_golden.npz"), **corr)

    # FFTAnalyzer with the windows the reference spells out
    ana = {}
    size = 1024
    s = rng.standard_normal(3 * size).astype(np.float32)
    ana["samples"] = s
    ana["w_flattop"] = flat_top(size)
    ana["w_kaiser6"] = kaiser(size, 6.0)
    ana["w_kaiser9"] = kaiser(size, 9.5)
    ana["w_rect"] = np.ones(size)
    for key in ["flattop", "kaiser6", "kaiser9", "rect"]:
        w = ana["w_" + key]
        ana["X0_" + key] = analyze(s, w)                # analyze(_:) of the first size samples
        ana["X1_" + key] = analyze(s, w, offset=size + 17)  # analyze(_:offset:)
    np.savez_compressed(os.path.join(HERE, "analyzer_golden.npz"), **ana)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
