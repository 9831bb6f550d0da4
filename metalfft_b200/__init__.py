"""metalfft_b200 -- B200 (sm_100a) implementation of MetalFFT's batched complex
FFT path, with the reference's Swift API mirrored in Python over the C ABI of
libmfft.so (include/mfft.h).

Reference API (docs/MetalFFT.swiftinterface:12-266) and its mirror here:

  MetalFFT(size:)                  -> MetalFFT(size)
    .forward(_:)                   -> .forward(x)
    .forward(input:output:)        -> .forward_into(x, out)
    .forward(batch:)               -> .forward_batch(xs)
    .inverse(_:)                   -> .inverse(x)
    (no counterpart: adjoints)     -> .backward(g, direction) / .backward_batch(gs, direction)
  MultiChannelFFT(channels:size:)  -> MultiChannelFFT(channels, size)
  Convolver(kernel:fftSize:)       -> Convolver(kernel, fft_size)
    .apply(to:) / blockSize / hopSize / recommendedFFTSize(forKernelCount:)
  FusedConvolver(kernel:fftSize:)  -> FusedConvolver(kernel, fft_size=4096)
  Correlator(fftSize:)             -> Correlator(fft_size) .cross(a, b) .auto(x)
  FFTAnalyzer(size:sampleRate:window:) -> FFTAnalyzer(size, sample_rate, window)
    .analyze(_:) / .analyze(_:offset:) -> AnalysisResult
  STFT(fftSize:hopSize:window:sampleRate:) -> STFT(fft_size, hop_size, window, sample_rate)
    .analyze(_:) / .spectrogram(_:) / frameCount(for:) -> STFTFrames / dB array / frame_count
  PSD.welch / PSD.coherence        -> PSD.welch / PSD.coherence (one launch for all frames)
  PSD.crossSpectral(channels:...)  -> PSD.cross_spectral(channels, fft_size, hop_size, ...)
  FFTError                         -> FFTError (same cases, Python exception)

Host arrays (numpy, lists) follow the Swift arrays' copy-in / copy-out
semantics.  torch CUDA tensors are transformed in device memory on the current
torch stream without any host copy.  Every call goes through libmfft.so; there
is no CPU path.
"""
import ctypes

import numpy as np

from . import _lib

__all__ = [
    "FFTError", "MetalFFT", "MultiChannelFFT", "Convolver", "FusedConvolver", "Correlator",
    "FFTAnalyzer", "AnalysisResult", "WindowType", "MixedBatch", "SARParameters", "SARTarget",
    "SARPipeline", "STFT", "STFTFrames", "PSD", "SpectralEstimator", "CrossSpectralResult",
    "COHERENCE_PER_FRAME", "COHERENCE_WELCH", "to_decibels", "lib", "shared_context",
]

lib = _lib.load()

HOST, DEVICE = 0, 1
FORWARD, INVERSE = -1, 1
TC_FP16_SPLIT3, TC_BF16 = 1, 2

# FFTError cases (Sources/MetalFFT/Internal/MetalContext.swift:6-30) by status
_CASES = {
    1: "noMetalDevice", 2: "noCommandQueue", 3: "libraryBuildFailed", 4: "kernelNotFound",
    5: "commandBufferFailed", 6: "invalidInputSize", 7: "batchInputSize",
    8: "unsupportedFFTSize", 9: "bufferAllocationFailed", 10: "invalidArgument",
    11: "timeout",
}


class FFTError(Exception):
    """Mirror of the reference's FFTError enum; `case` names the Swift case and
    `expected` / `got` / `batch_index` carry its associated values."""

    def __init__(self, status, message, expected=-1, got=-1, batch_index=-1):
        super().__init__(message)
        self.status = status
        self.case = _CASES.get(status, "unknown")
        self.expected = expected
        self.got = got
        self.batch_index = batch_index


def _raise(status):
    buf = ctypes.create_string_buffer(512)
    lib.mfft_last_error(buf, 512)
    e, g, i = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    lib.mfft_last_error_detail(ctypes.byref(e), ctypes.byref(g), ctypes.byref(i))
    raise FFTError(status, buf.value.decode() or lib.mfft_status_string(status).decode(),
                   e.value, g.value, i.value)


def _check(status):
    if status != 0:
        _raise(status)


def _fail(status, message, expected=-1, got=-1, batch_index=-1):
    raise FFTError(status, message, expected, got, batch_index)


_shared = None


def shared_context():
    """The process-wide context of the current CUDA device (MetalContext.shared())."""
    global _shared
    if _shared is None:
        h = ctypes.c_void_p()
        _check(lib.mfft_context_shared(ctypes.byref(h)))
        _shared = h
    return _shared


def _is_cuda_tensor(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _stream_of(t):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _host_c64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.complex64))


class MetalFFT:
    """Complex FFT of one size: forward (unscaled, e^{-2*pi*i*jk/n}) and
    inverse (1/n scaled).  Sizes: powers of two 64 ... 2^20 (the reference
    stops at 16384).  Not thread-safe (MetalFFT.swift:9)."""

    def __init__(self, size, context=None):
        self.size = int(size)
        self._ctx = context if context is not None else shared_context()
        h = ctypes.c_void_p()
        _check(lib.mfft_plan_create(self._ctx, self.size, ctypes.byref(h)))
        self._plan = h

    def __del__(self):
        p = getattr(self, "_plan", None)
        if p and lib is not None:
            lib.mfft_plan_destroy(p)
            self._plan = None

    @property
    def kernel_info(self):
        r, f, t, s = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib.mfft_plan_kernel_info(self._plan, ctypes.byref(r), ctypes.byref(f), ctypes.byref(t),
                                         ctypes.byref(s)))
        return {"radix": r.value, "lines_per_cta": f.value, "threads": t.value, "stages": s.value}

    def set_kernel(self, radix, lines_per_cta, stages=0):
        _check(lib.mfft_plan_set_kernel(self._plan, radix, lines_per_cta, stages))

    @staticmethod
    def variants(n):
        """Registered (radix, lines_per_cta, stages) variants for size n."""
        r = (ctypes.c_int * 64)()
        f = (ctypes.c_int * 64)()
        s = (ctypes.c_int * 64)()
        m = lib.mfft_list_kernels(n, r, f, s, 64)
        return [(r[i], f[i], s[i]) for i in range(min(m, 64))]

    # ---- four-step split (n > 16384) ---------------------------------------
    @property
    def split(self):
        """(n1, n2) of a four-step plan, (0, 0) for n <= 16384."""
        n1, n2 = ctypes.c_int64(), ctypes.c_int64()
        _check(lib.mfft_plan_split(self._plan, ctypes.byref(n1), ctypes.byref(n2)))
        return n1.value, n2.value

    def set_split(self, n1):
        """Pin the plan to n = n1 x n/n1 (64 <= n1 <= 1024, 128 <= n/n1 <= 1024)."""
        _check(lib.mfft_plan_set_split(self._plan, int(n1)))

    def autotune_split(self, batch=0):
        """Time every admissible split over `batch` transforms, keep the fastest, return n1."""
        n1 = ctypes.c_int()
        _check(lib.mfft_autotune_fourstep(self._plan, int(batch), ctypes.byref(n1)))
        return n1.value

    @staticmethod
    def splits(n):
        """Admissible four-step n1 values for size n ([] for n <= 16384)."""
        buf = (ctypes.c_int64 * 8)()
        m = lib.mfft_list_splits(int(n), buf, 8)
        return [buf[i] for i in range(min(m, 8))]

    # ---- raw entry ---------------------------------------------------------
    def exec(self, inp, out, batch, direction=FORWARD, tc_variant=0):
        """Run on device tensors (torch, complex64, contiguous): out = FFT(inp)."""
        if tc_variant:
            st = lib.mfft_exec_c2c_tc(self._plan, ctypes.c_void_p(inp.data_ptr()),
                                      ctypes.c_void_p(out.data_ptr()), batch, direction,
                                      tc_variant, DEVICE, _stream_of(inp))
        else:
            st = lib.mfft_exec_c2c(self._plan, ctypes.c_void_p(inp.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), batch, direction, DEVICE,
                                   _stream_of(inp))
        _check(st)
        return out

    def exec_backward(self, grad_out, grad_in, batch, direction=FORWARD):
        """Adjoint of exec on device tensors: grad_in = dL/dx for a real loss
        L of y = exec(x, direction), given grad_out = dL/dy (complex gradient
        dL/dRe + i dL/dIm).  FORWARD: n * inverse(grad_out); INVERSE:
        forward(grad_out) / n."""
        _check(lib.mfft_exec_c2c_backward(self._plan, ctypes.c_void_p(grad_out.data_ptr()),
                                          ctypes.c_void_p(grad_in.data_ptr()), batch, direction, DEVICE,
                                          _stream_of(grad_out)))
        return grad_in

    def backward(self, grad, direction=FORWARD):
        """Gradient with respect to the input of forward(_:) (direction
        FORWARD) or inverse(_:) (INVERSE) of one line."""
        self._check_len(grad)
        return self._run_backward(grad, 1, direction)

    def backward_batch(self, grads, direction=FORWARD):
        """backward of forward(batch:) / the batched inverse: one launch."""
        a, b = self._batch_array(grads)
        if b == 0:
            return np.empty((0, self.size), np.complex64)
        return self._run_backward(a, b, direction)

    def _run_backward(self, g, batch, direction):
        if _is_cuda_tensor(g):
            import torch
            if g.dtype != torch.complex64:
                _fail(10, "expected a complex64 tensor, got %s" % g.dtype)
            g = g.contiguous()
            return self.exec_backward(g, torch.empty_like(g), batch, direction)
        a = _host_c64(g)
        out = np.empty_like(a)
        _check(lib.mfft_exec_c2c_backward(self._plan, a.ctypes.data, out.ctypes.data, batch, direction, HOST,
                                          None))
        return out

    def forward_real(self, x):
        """Real input, n/2 + 1 complex bins per line (rfft): host arrays
        ([batch,] n) or a CUDA float32 tensor."""
        return self._real(x, True)

    def inverse_real(self, X):
        """n/2 + 1 bins per line -> n real samples (irfft, 1/n scaled)."""
        return self._real(X, False)

    def _real(self, x, forward):
        n, h = self.size, self.size // 2 + 1
        fn = lib.mfft_exec_r2c if forward else lib.mfft_exec_c2r
        if _is_cuda_tensor(x):
            import torch
            x = x.contiguous()
            batch = x.numel() // (n if forward else h)
            shape = x.shape[:-1] + ((h,) if forward else (n,))
            out = torch.empty(shape, dtype=torch.complex64 if forward else torch.float32, device=x.device)
            _check(fn(self._plan, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), batch, DEVICE,
                      _stream_of(x)))
            return out
        a = np.ascontiguousarray(np.asarray(x, dtype=np.float32 if forward else np.complex64))
        if a.shape[-1] != (n if forward else h):
            _fail(6, "expected last dimension %d, got %d" % (n if forward else h, a.shape[-1]),
                  n if forward else h, a.shape[-1])
        batch = a.size // a.shape[-1]
        out = np.empty(a.shape[:-1] + ((h,) if forward else (n,)), np.complex64 if forward else np.float32)
        _check(fn(self._plan, a.ctypes.data, out.ctypes.data, batch, HOST, None))
        return out

    def capture(self, calls):
        """One CUDA graph of device-tensor execs.  `calls` is a list of
        (inp, out, batch, direction) or (inp, out, batch, direction,
        tc_variant); the returned torch.cuda.CUDAGraph re-runs all of them
        with one replay(), so a small batch costs one graph launch instead of
        one host call per kernel.  The tensors must stay alive and in place."""
        import torch
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for c in calls:
                self.exec(*c)
        return g

    def _run(self, x, batch, direction, tc_variant=0):
        if _is_cuda_tensor(x):
            import torch
            if x.dtype != torch.complex64:
                _fail(10, "expected a complex64 tensor, got %s" % x.dtype)
            x = x.contiguous()
            out = torch.empty_like(x)
            return self.exec(x, out, batch, direction, tc_variant)
        a = _host_c64(x)
        out = np.empty_like(a)
        if tc_variant:
            st = lib.mfft_exec_c2c_tc(self._plan, a.ctypes.data, out.ctypes.data, batch, direction,
                                      tc_variant, HOST, None)
        else:
            st = lib.mfft_exec_c2c(self._plan, a.ctypes.data, out.ctypes.data, batch, direction,
                                   HOST, None)
        _check(st)
        return out

    def _check_len(self, x):
        n = x.numel() if _is_cuda_tensor(x) else len(x)
        if n != self.size:
            _fail(6, "Input size mismatch: expected %d, got %d" % (self.size, n), self.size, n)

    # ---- Swift API ---------------------------------------------------------
    def forward(self, x):
        """forward(_:) -- MetalFFT.swift:69-85."""
        self._check_len(x)
        return self._run(x, 1, FORWARD)

    def forward_into(self, x, out):
        """forward(input:output:) -- MetalFFT.swift:88-104 (out resized if needed)."""
        self._check_len(x)
        y = self._run(x, 1, FORWARD)
        if len(out) != self.size:
            out.resize(self.size, refcheck=False)
        out[...] = y
        return out

    def inverse(self, x):
        """inverse(_:) -- MetalFFT.swift:56-65: (1/n) conj(FFT(conj(X)))."""
        self._check_len(x)
        return self._run(x, 1, INVERSE)

    def _batch_array(self, xs):
        if _is_cuda_tensor(xs):
            if xs.dim() != 2 or xs.shape[1] != self.size:
                got = xs.shape[-1] if xs.dim() else 0
                _fail(7, "Batch element 0: expected %d, got %d" % (self.size, got), self.size, got, 0)
            return xs, xs.shape[0]
        if isinstance(xs, np.ndarray) and xs.ndim == 2:
            if xs.shape[1] != self.size:
                _fail(7, "Batch element 0: expected %d, got %d" % (self.size, xs.shape[1]),
                      self.size, xs.shape[1], 0)
            return _host_c64(xs), xs.shape[0]
        for i, el in enumerate(xs):
            if len(el) != self.size:
                _fail(7, "Batch element %d: expected %d, got %d" % (i, self.size, len(el)),
                      self.size, len(el), i)
        if len(xs) == 0:
            return None, 0
        return _host_c64(np.stack([np.asarray(el) for el in xs])), len(xs)

    def forward_batch(self, xs, tc_variant=0):
        """forward(batch:) -- MetalFFT.swift:108-133; one launch for the batch."""
        a, b = self._batch_array(xs)
        if b == 0:
            return np.empty((0, self.size), np.complex64)
        return self._run(a, b, FORWARD, tc_variant)

    def inverse_batch(self, xs, tc_variant=0):
        a, b = self._batch_array(xs)
        if b == 0:
            return np.empty((0, self.size), np.complex64)
        return self._run(a, b, INVERSE, tc_variant)


class MultiChannelFFT:
    """MultiChannelFFT (MultiChannelFFT.swift:19-54): channels x size in one launch."""

    def __init__(self, channels, size):
        if channels <= 0:
            _fail(10, "channels must be > 0")
        self.channels = int(channels)
        self.size = int(size)
        self._fft = MetalFFT(size)

    def _check(self, xs):
        n = xs.shape[0] if hasattr(xs, "shape") else len(xs)
        if n != self.channels:
            _fail(10, "Expected %d channels, got %d" % (self.channels, n))

    def forward(self, xs):
        self._check(xs)
        return self._fft.forward_batch(xs)

    def inverse(self, xs):
        self._check(xs)
        return self._fft.inverse_batch(xs)


from ._dsp import (AnalysisResult, Convolver, Correlator, FFTAnalyzer, FusedConvolver,  # noqa: E402
                   MixedBatch, WindowType)
from ._sar import (RC_FP16, RC_FP32, SARParameters, SARPipeline, SARTarget, expected_bins,  # noqa: E402
                   point_target_metrics)
from ._spectral import (COHERENCE_PER_FRAME, COHERENCE_WELCH, PSD, STFT, CrossSpectralResult,  # noqa: E402
                        SpectralEstimator, STFTFrames, to_decibels)
