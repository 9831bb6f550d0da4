"""Mirrors of the reference's STFT and PSD (Sources/MetalFFT/DSP/STFT.swift,
DSP/PSD.swift) over libmfft's C ABI: every frame of a signal is windowed and
transformed in one launch instead of one FFT call per frame."""
import ctypes

import numpy as np

from . import DEVICE, HOST, _check, _fail, _is_cuda_tensor, _stream_of, lib, shared_context
from ._dsp import WindowType, _host_f32, _ptr


def to_decibels(magnitudes, floor_db=-120.0):
    """Spectrum.toDecibels (DSP/Spectrum.swift:47-55): vDSP_vdbcon with the
    amplitude flag, 20*log10(x), clipped below at floor_db."""
    m = np.asarray(magnitudes, dtype=np.float64)
    with np.errstate(divide="ignore"):
        db = 20.0 * np.log10(m)
    return np.maximum(db, floor_db).astype(np.float32)


class STFTFrames:
    """The frames of STFT.analyze (STFTFrame, STFT.swift:5-16) as arrays:
    complex (frames x fft_size), magnitudes = |X|^2, magnitudes_db, phase."""

    def __init__(self, complex_, magnitudes):
        self.complex = complex_
        self.magnitudes = magnitudes

    def __len__(self):
        return self.complex.shape[0]

    @property
    def magnitudes_db(self):
        return to_decibels(self.magnitudes)

    @property
    def phase(self):
        return np.angle(self.complex).astype(np.float32)


class _Spectral:
    def __init__(self, fft_size, hop_size, window=None, context=None):
        w = window if window is not None else WindowType(WindowType.HANN)
        if isinstance(w, int):
            w = WindowType(w)
        h = ctypes.c_void_p()
        _check(lib.mfft_spectral_create(context or shared_context(), int(fft_size), int(hop_size), w.kind,
                                        float(w.beta), ctypes.byref(h)))
        self._h = h
        self.fft_size = int(fft_size)
        self.hop_size = int(hop_size)

    def frame_count(self, sample_count):
        return int(lib.mfft_stft_frame_count(self._h, int(sample_count)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.mfft_spectral_destroy(h)
            self._h = None


class STFT(_Spectral):
    """STFT(fftSize:hopSize:window:sampleRate:) (STFT.swift:19-108)."""

    def __init__(self, fft_size, hop_size, window=None, sample_rate=1.0, context=None):
        super().__init__(fft_size, hop_size, window, context)
        self.sample_rate = float(sample_rate)

    def bin_frequency(self, b):
        return b * self.sample_rate / self.fft_size

    def frame_time(self, f):
        return f * self.hop_size / self.sample_rate

    def analyze(self, signal):
        """All frames: STFTFrames (host arrays), or for a CUDA float32 tensor a
        (spectra, power) pair of device tensors."""
        if _is_cuda_tensor(signal):
            import torch
            x = signal.contiguous()
            f = self.frame_count(x.numel())
            spec = torch.empty((f, self.fft_size), dtype=torch.complex64, device=x.device)
            power = torch.empty((f, self.fft_size), dtype=torch.float32, device=x.device)
            _check(lib.mfft_stft_analyze(self._h, _ptr(x), x.numel(), _ptr(spec), _ptr(power), DEVICE,
                                         _stream_of(x)))
            return spec, power
        x = _host_f32(signal)
        f = self.frame_count(len(x))
        spec = np.empty((f, self.fft_size), np.complex64)
        power = np.empty((f, self.fft_size), np.float32)
        _check(lib.mfft_stft_analyze(self._h, _ptr(x), len(x), _ptr(spec), _ptr(power), HOST, None))
        return STFTFrames(spec, power)

    def spectrogram(self, signal):
        """[time][frequency] dB magnitudes (STFT.swift:91-94)."""
        return self.analyze(signal).magnitudes_db


class CrossSpectralResult:
    """CrossSpectralResult (CrossSpectral.swift:11-38): power (C x fft),
    cross_spectra (P x fft complex, X_i conj(X_j)), coherence (P x fft), with
    pairs in upper-triangle order (0,1), (0,2), ..., (C-2, C-1)."""

    def __init__(self, channels, fft_size, power, cross_spectra, coherence):
        self.channels = channels
        self.fft_size = fft_size
        self.power = power
        self.cross_spectra = cross_spectra
        self.coherence = coherence

    @property
    def pair_count(self):
        return self.channels * (self.channels - 1) // 2

    def pair_index(self, i, j):
        """Flat pair index of channels i < j (CrossSpectral.swift:29-37)."""
        if not (0 <= i < j < self.channels):
            raise ValueError(f"pair_index needs 0 <= i < j < {self.channels}, got ({i}, {j})")
        return sum(self.channels - 1 - a for a in range(i)) + (j - i - 1)


COHERENCE_PER_FRAME, COHERENCE_WELCH = 0, 1


def _cross_spectral_call(h, fft, signals, coherence_mode):
    """signals: C x n (host array or CUDA float32 tensor)."""
    if _is_cuda_tensor(signals):
        import torch
        x = signals.contiguous()
        if x.dim() != 2:
            raise ValueError("signals must be channels x samples")
        c, n = x.shape
        p = c * (c - 1) // 2
        power = torch.empty((c, fft), dtype=torch.float32, device=x.device)
        cross = torch.empty((p, fft), dtype=torch.complex64, device=x.device)
        coh = torch.empty((p, fft), dtype=torch.float32, device=x.device)
        _check(lib.mfft_psd_cross_spectral(h, _ptr(x), c, n, _ptr(power), _ptr(cross) if p else None,
                                           _ptr(coh) if p else None, int(coherence_mode), DEVICE, _stream_of(x)))
        return power, cross, coh
    chans = [np.asarray(ch, dtype=np.float32).ravel() for ch in signals]
    if not chans or len(chans) > 16:
        _fail(10, "crossSpectral requires 1-16 channels", got=len(chans))
    if any(len(ch) != len(chans[0]) for ch in chans):
        _fail(10, "all channels must have the same length")
    x = np.ascontiguousarray(np.stack(chans))
    c, n = x.shape
    p = c * (c - 1) // 2
    power = np.empty((c, fft), np.float32)
    cross = np.empty((p, fft), np.complex64)
    coh = np.empty((p, fft), np.float32)
    _check(lib.mfft_psd_cross_spectral(h, _ptr(x), c, n, _ptr(power), _ptr(cross) if p else None,
                                       _ptr(coh) if p else None, int(coherence_mode), HOST, None))
    return power, cross, coh


class PSD:
    """PSD.welch, PSD.coherence (PSD.swift:6-134) and PSD.crossSpectral
    (CrossSpectral.swift:56-152)."""

    @staticmethod
    def welch(signal, fft_size, hop_size, sample_rate, window=None, context=None):
        s = _Spectral(fft_size, hop_size, window, context)
        out = np.empty(s.fft_size, np.float32)
        x = _host_f32(signal)
        _check(lib.mfft_psd_welch(s._h, _ptr(x), len(x), float(sample_rate), _ptr(out), HOST, None))
        return out

    @staticmethod
    def coherence(a, b, fft_size, hop_size, sample_rate=1.0, window=None, context=None):
        s = _Spectral(fft_size, hop_size, window, context)
        out = np.empty(s.fft_size, np.float32)
        xa, xb = _host_f32(a), _host_f32(b)
        _check(lib.mfft_psd_coherence(s._h, _ptr(xa), len(xa), _ptr(xb), len(xb), _ptr(out), HOST, None))
        return out

    @staticmethod
    def cross_spectral(channels, fft_size, hop_size, sample_rate=1.0, window=None, coherence_mode=COHERENCE_PER_FRAME,
                       context=None):
        """CrossSpectralResult of 1..16 equal-length real channels.
        coherence_mode COHERENCE_PER_FRAME is the reference's mean of per-frame
        |S_ij|^2 / (p_i p_j); COHERENCE_WELCH is |mean S_ij|^2 /
        (mean p_i mean p_j).  sample_rate labels bins only, as in the reference."""
        s = _Spectral(fft_size, hop_size, window, context)
        power, cross, coh = _cross_spectral_call(s._h, s.fft_size, channels, coherence_mode)
        return CrossSpectralResult(power.shape[0], s.fft_size, power, cross, coh)


class SpectralEstimator(_Spectral):
    """Reusable handle for repeated Welch / coherence estimates with one
    frame geometry and window (device tensors or host arrays)."""

    def welch(self, signal, sample_rate, out=None):
        if _is_cuda_tensor(signal):
            import torch
            x = signal.contiguous()
            out = out if out is not None else torch.empty(self.fft_size, dtype=torch.float32, device=x.device)
            _check(lib.mfft_psd_welch(self._h, _ptr(x), x.numel(), float(sample_rate), _ptr(out), DEVICE,
                                      _stream_of(x)))
            return out
        x = _host_f32(signal)
        res = np.empty(self.fft_size, np.float32)
        _check(lib.mfft_psd_welch(self._h, _ptr(x), len(x), float(sample_rate), _ptr(res), HOST, None))
        return res

    def coherence(self, a, b, out=None):
        if _is_cuda_tensor(a):
            import torch
            xa, xb = a.contiguous(), b.contiguous()
            out = out if out is not None else torch.empty(self.fft_size, dtype=torch.float32, device=xa.device)
            _check(lib.mfft_psd_coherence(self._h, _ptr(xa), xa.numel(), _ptr(xb), xb.numel(), _ptr(out), DEVICE,
                                          _stream_of(xa)))
            return out
        xa, xb = _host_f32(a), _host_f32(b)
        res = np.empty(self.fft_size, np.float32)
        _check(lib.mfft_psd_coherence(self._h, _ptr(xa), len(xa), _ptr(xb), len(xb), _ptr(res), HOST, None))
        return res

    def cross_spectral(self, signals, coherence_mode=COHERENCE_PER_FRAME):
        """(power, cross, coherence) of channels x samples: device tensors for
        a CUDA float32 tensor, host arrays otherwise."""
        return _cross_spectral_call(self._h, self.fft_size, signals, coherence_mode)
