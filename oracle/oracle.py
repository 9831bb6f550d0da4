"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() (as the
checker) and bench.py's CPU-baseline leg.  The product (metalfft_b200/) never
imports it.  See oracle.c for what each function restates.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_i64, _int, _dbl = ctypes.c_int64, ctypes.c_int, ctypes.c_double


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "mfo_max_threads": (_int, []),
            "mfo_dft_c128": (None, [_dp, _dp, _i64, _int]),
            "mfo_fft_c128": (None, [_dp, _dp, _i64, _i64, _int, _int]),
            "mfo_fft_c64_to_c128": (None, [_fp, _dp, _i64, _i64, _int, _int]),
            "mfo_rel_rms_c64_vs_c128": (_dbl, [_fp, _dp, _i64, _int]),
            "mfo_ref_fft_c64": (None, [_fp, _fp, _int, _i64, _int, _int]),
            "mfo_ref_fourstep_split": (None, [_int, ctypes.POINTER(_int), ctypes.POINTER(_int)]),
            "mfo_ref_conv_ola_f32": (None, [_fp, _i64, _fp, _int, _int, _fp, _int]),
            "mfo_conv_f64": (None, [_dp, _i64, _dp, _int, _int, _dp, _int]),
            "mfo_conv_adjoint_f64": (None, [_dp, _i64, _dp, _int, _dp, _dp, _dp]),
            "mfo_corr_f64": (None, [_dp, _i64, _dp, _i64, _int, _dp]),
            "mfo_ref_corr_f32": (None, [_fp, _i64, _fp, _i64, _int, _fp]),
            "mfo_window": (None, [_int, _int, _dbl, _dp]),
            "mfo_stft_frames": (_i64, [_i64, _int, _int]),
            "mfo_stft": (None, [_dp, _i64, _int, _int, _dp, _dp]),
            "mfo_welch": (_i64, [_dp, _i64, _int, _int, _dp, _dbl, _dp]),
            "mfo_coherence": (_i64, [_dp, _i64, _dp, _i64, _int, _int, _dp, _dp]),
            "mfo_cross_spectral": (_i64, [_dp, _int, _i64, _int, _int, _dp, _dp, _dp, _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _f(a):
    return a.ctypes.data_as(_fp)


def max_threads():
    return load().mfo_max_threads()


def dft(x, sign=-1):
    """Naive FP64 DFT of one line (exact index reduction)."""
    x = np.ascontiguousarray(x, np.complex128)
    out = np.empty_like(x)
    load().mfo_dft_c128(_d(x), _d(out), x.size, sign)
    return out


def fft64(x, sign=-1, threads=0):
    """FP64 FFT of each row of x (complex128), unscaled."""
    x = np.ascontiguousarray(x, np.complex128)
    n = x.shape[-1]
    out = np.empty_like(x)
    load().mfo_fft_c128(_d(x), _d(out), n, x.size // n, sign, threads)
    return out


def truth(x64, inverse=False, threads=0):
    """FP64 ground truth for complex64 rows: forward, or inverse with 1/n."""
    x64 = np.ascontiguousarray(x64, np.complex64)
    n = x64.shape[-1]
    out = np.empty(x64.shape, np.complex128)
    load().mfo_fft_c64_to_c128(_f(x64), _d(out), n, x64.size // n, +1 if inverse else -1, threads)
    if inverse:
        out /= n
    return out


def rel_rms(y, ref, threads=0):
    """||y - ref|| / ||ref|| in FP64 (MetalFFTTests.swift:190-198 definition)."""
    y = np.ascontiguousarray(y, np.complex64)
    ref = np.ascontiguousarray(ref, np.complex128)
    return load().mfo_rel_rms_c64_vs_c128(_f(y), _d(ref), y.size, threads)


def ref_fft(x, inverse=False, threads=0):
    """FP32 restatement of the reference's Stockham / four-step path."""
    x = np.ascontiguousarray(x, np.complex64)
    n = x.shape[-1]
    out = np.empty_like(x)
    load().mfo_ref_fft_c64(_f(x), _f(out), n, x.size // n, 1 if inverse else 0, threads)
    return out


def ref_fourstep_split(n):
    a, b = _int(), _int()
    load().mfo_ref_fourstep_split(n, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def ref_conv(x, h, fft, threads=0):
    x = np.ascontiguousarray(x, np.float32)
    h = np.ascontiguousarray(h, np.float32)
    y = np.empty(len(x) + len(h) - 1, np.float32)
    load().mfo_ref_conv_ola_f32(_f(x), len(x), _f(h), len(h), fft, _f(y), threads)
    return y


def conv64(x, h, fft, threads=0):
    x = np.ascontiguousarray(x, np.float64)
    h = np.ascontiguousarray(h, np.float64)
    y = np.empty(len(x) + len(h) - 1, np.float64)
    load().mfo_conv_f64(_d(x), len(x), _d(h), len(h), fft, _d(y), threads)
    return y


def conv_adjoint64(x, h, g):
    x = np.ascontiguousarray(x, np.float64)
    h = np.ascontiguousarray(h, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    dx = np.empty(len(x), np.float64)
    dh = np.empty(len(h), np.float64)
    load().mfo_conv_adjoint_f64(_d(x), len(x), _d(h), len(h), _d(g), _d(dx), _d(dh))
    return dx, dh


def corr64(a, b, fft):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    r = np.empty(fft, np.float64)
    load().mfo_corr_f64(_d(a), len(a), _d(b), len(b), fft, _d(r))
    return r


def ref_corr(a, b, fft):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    r = np.empty(fft, np.float32)
    load().mfo_ref_corr_f32(_f(a), len(a), _f(b), len(b), fft, _f(r))
    return r


def window(kind, n, beta=6.0):
    w = np.empty(n, np.float64)
    load().mfo_window(kind, n, beta, _d(w))
    return w


def stft_frames(n, fft, hop):
    return load().mfo_stft_frames(n, fft, hop)


def stft64(x, fft, hop, w):
    """FP64 STFT (frames x fft complex128) of real x with window w."""
    x = np.ascontiguousarray(x, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    out = np.empty((stft_frames(len(x), fft, hop), fft), np.complex128)
    load().mfo_stft(_d(x), len(x), fft, hop, _d(w), _d(out))
    return out


def welch64(x, fft, hop, w, sample_rate):
    x = np.ascontiguousarray(x, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    out = np.empty(fft, np.float64)
    load().mfo_welch(_d(x), len(x), fft, hop, _d(w), sample_rate, _d(out))
    return out


def coherence64(a, b, fft, hop, w):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    out = np.empty(fft, np.float64)
    load().mfo_coherence(_d(a), len(a), _d(b), len(b), fft, hop, _d(w), _d(out))
    return out


def cross_spectral64(x, fft, hop, w):
    """FP64 PSD.crossSpectral of channels x n real samples: (power C x fft,
    cross P x fft complex128, per-frame-averaged coherence P x fft)."""
    x = np.ascontiguousarray(x, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    c, n = x.shape
    p = c * (c - 1) // 2
    power = np.empty((c, fft), np.float64)
    cross = np.zeros((max(p, 1), fft), np.complex128)
    coh = np.zeros((max(p, 1), fft), np.float64)
    load().mfo_cross_spectral(_d(x), c, n, fft, hop, _d(w), _d(power), _d(cross), _d(coh))
    return power, cross[:p], coh[:p]


# ---- seeded generators shared by tests, smoke and bench ---------------------

def uniform_c64(shape, seed, lo=-1.0, hi=1.0):
    """re, im i.i.d. U[lo, hi) (the reference's Float.random(in: -1...1))."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(lo, hi, size=tuple(shape) + (2,)).astype(np.float32)
    return z.view(np.complex64)[..., 0]


def normal_c64(shape, seed):
    rng = np.random.default_rng(seed)
    z = rng.standard_normal(size=tuple(shape) + (2,), dtype=np.float32)
    return z.view(np.complex64)[..., 0]


# ---- SAR (sar_oracle.c) -------------------------------------------------------

class _SarParams(ctypes.Structure):
    _fields_ = [("pulses", ctypes.c_int64), ("range_n", ctypes.c_int64), ("chirp_samples", ctypes.c_int64),
                ("bandwidth", ctypes.c_double), ("sample_rate", ctypes.c_double), ("prf", ctypes.c_double),
                ("velocity", ctypes.c_double), ("carrier", ctypes.c_double), ("center_range", ctypes.c_double)]


class _SarTarget(ctypes.Structure):
    _fields_ = [("range_m", ctypes.c_double), ("azimuth_m", ctypes.c_double), ("amplitude", ctypes.c_double),
                ("phase", ctypes.c_double)]


def _sar_args(params, targets):
    p = _SarParams(*(getattr(params, f) for f, _ in _SarParams._fields_))
    arr = (_SarTarget * max(1, len(targets)))(*[_SarTarget(t.range_m, t.azimuth_m, t.amplitude, t.phase)
                                                  for t in targets])
    return p, arr


def sar_simulate(params, targets, snr_db, seed):
    L = load()
    L.mfo_sar_simulate.restype = None
    p, arr = _sar_args(params, targets)
    raw = np.empty((params.pulses, params.range_n), np.complex128)
    L.mfo_sar_simulate(ctypes.byref(p), arr, len(targets), ctypes.c_double(snr_db), ctypes.c_uint64(seed),
                       raw.ctypes.data_as(_dp))
    return raw


def sar_image(params, raw, chirp, phi):
    L = load()
    L.mfo_sar_image.restype = None
    p, _ = _sar_args(params, [])
    raw = np.ascontiguousarray(raw, np.complex128)
    ch = np.ascontiguousarray(chirp, np.complex128)
    ph = np.ascontiguousarray(phi, np.float64)
    img = np.empty((params.pulses, params.range_n), np.complex128)
    L.mfo_sar_image(ctypes.byref(p), raw.ctypes.data_as(_dp), ch.ctypes.data_as(_dp), ph.ctypes.data_as(_dp),
                    img.ctypes.data_as(_dp), None)
    return img


def sar_loss_grad(params, raw, chirp, phi):
    L = load()
    L.mfo_sar_loss_grad.restype = ctypes.c_double
    p, _ = _sar_args(params, [])
    raw = np.ascontiguousarray(raw, np.complex128)
    ch = np.ascontiguousarray(chirp, np.complex128)
    ph = np.ascontiguousarray(phi, np.float64)
    d = np.empty(params.pulses, np.float64)
    loss = L.mfo_sar_loss_grad(ctypes.byref(p), raw.ctypes.data_as(_dp), ch.ctypes.data_as(_dp),
                               ph.ctypes.data_as(_dp), d.ctypes.data_as(_dp))
    return loss, d


def sar_focus(params, rd, reference_signs=False):
    """FP64 focusing (RCMC + azimuth matched filter + azimuth inverse FFT) of
    a range-Doppler image (pulses x range_n, Doppler-major)."""
    L = load()
    L.mfo_sar_focus.restype = None
    p, _ = _sar_args(params, [])
    rd = np.ascontiguousarray(rd, np.complex128)
    out = np.empty_like(rd)
    L.mfo_sar_focus(ctypes.byref(p), rd.ctypes.data_as(_dp), int(bool(reference_signs)), out.ctypes.data_as(_dp))
    return out
