"""Mirrors of the reference's FFT callers (Convolver, FusedConvolver,
Correlator, FFTAnalyzer) and the mixed-size batch, over libmfft's C ABI."""
import ctypes
import math

import numpy as np

from . import (DEVICE, FORWARD, HOST, FFTError, _check, _fail, _is_cuda_tensor, _stream_of, lib,
               shared_context)


def _host_f32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


def _ptr(x):
    if x is None:
        return None
    if _is_cuda_tensor(x):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(x.ctypes.data)


class Convolver:
    """FFT-based overlap-add FIR convolution (Convolve.swift:8-87).

    The B200 path runs every block's FFT -> * H -> inverse -> overlap-add in one
    fused launch per call (not one GPU round trip per block).  fft_size must
    be a power of two 64 .. 16384 and > len(kernel)."""

    def __init__(self, kernel, fft_size, context=None):
        k = _host_f32(kernel)
        if not fft_size > len(k):
            _fail(10, "fftSize must be > kernel.count; got fftSize=%d, kernel.count=%d"
                  % (fft_size, len(k)))
        h = ctypes.c_void_p()
        _check(lib.mfft_conv_create(context or shared_context(), k.ctypes.data, len(k),
                                    int(fft_size), ctypes.byref(h)))
        self._h = h
        self.block_size = int(lib.mfft_conv_block_size(h))
        self.hop_size = int(lib.mfft_conv_hop_size(h))
        self.kernel_len = len(k)

    # Swift spellings
    @property
    def blockSize(self):  # noqa: N802
        return self.block_size

    @property
    def hopSize(self):  # noqa: N802
        return self.hop_size

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.mfft_conv_destroy(h)
            self._h = None

    @staticmethod
    def recommended_fft_size(kernel_count):
        """recommendedFFTSize(forKernelCount:) (Convolve.swift:83-86); None if none."""
        s = int(lib.mfft_recommended_fft_size(int(kernel_count)))
        return s or None

    def apply(self, signal):
        """apply(to:) -- output length len(signal) + len(kernel) - 1."""
        if _is_cuda_tensor(signal):
            import torch
            x = signal.contiguous()
            out = torch.empty(x.numel() + self.kernel_len - 1, dtype=torch.float32, device=x.device)
            _check(lib.mfft_conv_apply(self._h, _ptr(x), x.numel(), _ptr(out), DEVICE, _stream_of(x)))
            return out
        x = _host_f32(signal)
        out = np.empty(len(x) + self.kernel_len - 1, np.float32)
        _check(lib.mfft_conv_apply(self._h, _ptr(x), len(x), _ptr(out), HOST, None))
        return out

    def backward(self, signal, grad_out):
        """Gradients of a loss w.r.t. signal and kernel given dL/d(apply(signal))."""
        if _is_cuda_tensor(signal):
            import torch
            x = signal.contiguous()
            g = grad_out.contiguous()
            dx = torch.empty_like(x)
            dh = torch.empty(self.kernel_len, dtype=torch.float32, device=x.device)
            _check(lib.mfft_conv_backward(self._h, _ptr(x), x.numel(), _ptr(g), _ptr(dx), _ptr(dh),
                                          DEVICE, _stream_of(x)))
            return dx, dh
        x = _host_f32(signal)
        g = _host_f32(grad_out)
        if len(g) != len(x) + self.kernel_len - 1:
            _fail(6, "grad_out: expected %d, got %d" % (len(x) + self.kernel_len - 1, len(g)),
                  len(x) + self.kernel_len - 1, len(g))
        dx = np.empty_like(x)
        dh = np.empty(self.kernel_len, np.float32)
        _check(lib.mfft_conv_backward(self._h, _ptr(x), len(x), _ptr(g), _ptr(dx), _ptr(dh), HOST,
                                      None))
        return dx, dh


class FusedConvolver(Convolver):
    """FusedConvolver (FusedConvolver.swift:17-134): the reference's single
    dispatch FFT * H IFFT per block, fftSize 4096, with its Precision modes
    (:27-36) by their Swift case names: "float32" (default), "float16Pure",
    "float16Storage", "float16Mixed"."""

    supported_size = 4096
    PRECISIONS = {"float32": 0, "float16Pure": 1, "float16Storage": 2, "float16Mixed": 3}

    def __init__(self, kernel, fft_size=4096, precision="float32", context=None):
        if fft_size != self.supported_size:
            _fail(10, "FusedConvolver only supports fftSize=%d" % self.supported_size)
        if precision not in self.PRECISIONS:
            _fail(10, "unknown FusedConvolver precision %r (one of %s)" % (precision, ", ".join(self.PRECISIONS)))
        super().__init__(kernel, fft_size, context)
        _check(lib.mfft_conv_set_precision(self._h, self.PRECISIONS[precision]))
        self.precision = precision


class Correlator:
    """Circular cross / auto correlation via FFT (Correlate.swift:7-62)."""

    def __init__(self, fft_size, context=None):
        h = ctypes.c_void_p()
        _check(lib.mfft_corr_create(context or shared_context(), int(fft_size), ctypes.byref(h)))
        self._h = h
        self.fft_size = int(fft_size)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.mfft_corr_destroy(h)
            self._h = None

    def cross(self, a, b):
        a = _host_f32(a)
        b = _host_f32(b)
        out = np.empty(self.fft_size, np.float32)
        _check(lib.mfft_corr_cross(self._h, _ptr(a), len(a), _ptr(b), len(b), _ptr(out), HOST, None))
        return out

    def auto(self, x):
        return self.cross(x, x)


class WindowType:
    """WindowType (Window.swift:6-24)."""
    HANN, HAMMING, BLACKMAN, FLAT_TOP, KAISER, RECTANGULAR = range(6)

    def __init__(self, kind, beta=6.0):
        self.kind = kind
        self.beta = beta

    @classmethod
    def kaiser(cls, beta):
        return cls(cls.KAISER, beta)

    def coefficients(self, size):
        out = np.empty(size, np.float32)
        _check(lib.mfft_window(self.kind, size, float(self.beta), out.ctypes.data))
        return out


class AnalysisResult:
    """AnalysisResult (FFTAnalyzer.swift:6-62): lazy views of one spectrum."""

    def __init__(self, complex_, sample_rate, fft_size):
        self.complex = complex_
        self.sample_rate = sample_rate
        self.fft_size = fft_size

    @property
    def magnitudes(self):
        c = np.asarray(self.complex)
        return (c.real * c.real + c.imag * c.imag).astype(np.float32)

    @property
    def magnitudes_db(self):
        return (10.0 * np.log10(np.maximum(self.magnitudes, 1e-12))).astype(np.float32)

    @property
    def phase(self):
        return np.angle(np.asarray(self.complex)).astype(np.float32)

    def bin_frequency(self, b):
        return b * self.sample_rate / self.fft_size

    @property
    def rms(self):
        return float(math.sqrt(float(np.sum(self.magnitudes, dtype=np.float64))) / self.fft_size)


class FFTAnalyzer:
    """window -> FFT -> AnalysisResult (FFTAnalyzer.swift:68-117), windowing
    fused into the FFT's load on the device."""

    def __init__(self, size, sample_rate, window=None, context=None):
        w = window if window is not None else WindowType(WindowType.HANN)
        if isinstance(w, int):
            w = WindowType(w)
        h = ctypes.c_void_p()
        _check(lib.mfft_analyzer_create(context or shared_context(), int(size), float(sample_rate),
                                        w.kind, float(w.beta), ctypes.byref(h)))
        self._h = h
        self.size = int(size)
        self.sample_rate = float(sample_rate)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.mfft_analyzer_destroy(h)
            self._h = None

    def analyze(self, samples, offset=None):
        x = _host_f32(samples)
        if offset is None:
            if len(x) != self.size:
                _fail(10, "samples.count must equal size (%d), got %d" % (self.size, len(x)))
            offset = 0
        out = np.empty(self.size, np.complex64)
        _check(lib.mfft_analyzer_analyze(self._h, _ptr(x), len(x), int(offset), out.ctypes.data, HOST,
                                         None))
        return AnalysisResult(out, self.sample_rate, self.size)


class _Desc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("count", ctypes.c_int64), ("offset", ctypes.c_int64)]


class MixedBatch:
    """Transforms of several sizes in one persistent launch that draws its
    work items from a device-side queue (no reference counterpart).
    sizes_counts: [(n, count), ...];
    transforms of a class are stored back to back, classes one after another
    in the given order."""

    def __init__(self, sizes_counts, context=None):
        descs = (_Desc * len(sizes_counts))()
        off = 0
        for i, (n, c) in enumerate(sizes_counts):
            descs[i].n, descs[i].count, descs[i].offset = int(n), int(c), off
            off += int(n) * int(c)
        h = ctypes.c_void_p()
        _check(lib.mfft_multi_create(context or shared_context(), ctypes.cast(descs, ctypes.c_void_p),
                                     len(sizes_counts), ctypes.byref(h)))
        self._h = h
        self.points = int(lib.mfft_multi_points(h))
        self.layout = [(int(d.n), int(d.count), int(d.offset)) for d in descs]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.mfft_multi_destroy(h)
            self._h = None

    def exec(self, inp, out, direction=FORWARD):
        """Device tensors (torch complex64, `points` elements)."""
        _check(lib.mfft_multi_exec(self._h, _ptr(inp), _ptr(out), direction, DEVICE, _stream_of(inp)))
        return out

    def capture(self, inp, out, direction=FORWARD):
        """One CUDA graph of exec(inp, out, direction): every launch of the
        batch replays with one graph launch.  The tensors must stay alive and
        in place."""
        import torch
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.exec(inp, out, direction)
        return g

    def forward(self, x):
        if _is_cuda_tensor(x):
            import torch
            out = torch.empty_like(x)
            return self.exec(x.contiguous(), out)
        a = np.ascontiguousarray(np.asarray(x, np.complex64))
        if a.size != self.points:
            raise FFTError(6, "expected %d points, got %d" % (self.points, a.size), self.points, a.size)
        out = np.empty_like(a)
        _check(lib.mfft_multi_exec(self._h, _ptr(a), _ptr(out), FORWARD, HOST, None))
        return out
