"""SAR range-Doppler chain over libmfft's C ABI: the B200 form of the
reference's RDAFusedPipeline (src/radar/rda_fused_pipeline.swift) with FP16
storage, plus its simulator (src/radar/sar_simulator.swift) and the adjoint
of the sharpness loss with respect to a per-pulse phase."""
import ctypes

import numpy as np

from . import _check, lib, shared_context


class SARParameters(ctypes.Structure):
    """SARParameters (sar_simulator.swift:22-67); see mfft_sar_params."""
    _fields_ = [("pulses", ctypes.c_int64), ("range_n", ctypes.c_int64), ("chirp_samples", ctypes.c_int64),
                ("bandwidth", ctypes.c_double), ("sample_rate", ctypes.c_double), ("prf", ctypes.c_double),
                ("velocity", ctypes.c_double), ("carrier", ctypes.c_double), ("center_range", ctypes.c_double)]

    @classmethod
    def default(cls, pulses=4096, range_n=8192, chirp_samples=1024, tbp=512.0):
        p = cls()
        _check(lib.mfft_sar_default_params(pulses, range_n, chirp_samples, float(tbp), ctypes.byref(p)))
        return p

    def chirp_reference(self):
        out = np.empty(self.range_n, np.complex64)
        _check(lib.mfft_sar_chirp_reference(ctypes.byref(self), out.ctypes.data))
        return out

    @property
    def tau0(self):
        return 2.0 * self.center_range / 299792458.0 - (self.range_n // 2) / self.sample_rate


class SARTarget(ctypes.Structure):
    _fields_ = [("range_m", ctypes.c_double), ("azimuth_m", ctypes.c_double), ("amplitude", ctypes.c_double),
                ("phase", ctypes.c_double)]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(t):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


class SARPipeline:
    """Range compression -> corner turn -> azimuth FFT on device tensors."""

    def __init__(self, params, chirp=None, context=None):
        self.params = params
        c = np.ascontiguousarray(chirp if chirp is not None else params.chirp_reference(), np.complex64)
        self._ctx = context or shared_context()
        h = ctypes.c_void_p()
        _check(lib.mfft_sar_create(self._ctx, ctypes.byref(params), c.ctypes.data, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.mfft_sar_destroy(h)
            self._h = None

    @property
    def shape(self):
        return (self.params.pulses, self.params.range_n)

    def simulate(self, targets, snr_db, seed):
        """SARSimulator.simulate on the device -> complex64 (pulses, range_n)."""
        import torch
        arr = (SARTarget * max(1, len(targets)))(*targets)
        raw = torch.empty(self.shape, dtype=torch.complex64, device="cuda")
        _check(lib.mfft_sar_simulate(self._ctx, ctypes.byref(self.params), ctypes.cast(arr, ctypes.c_void_p),
                                     len(targets), float(snr_db), int(seed), _p(raw), _stream(raw)))
        return raw

    def quantize(self, raw):
        """FP16 storage with one power-of-two scale per pulse."""
        import torch
        na, nr = self.shape
        h = torch.empty((na, nr, 2), dtype=torch.float16, device=raw.device)
        sc = torch.empty(na, dtype=torch.float32, device=raw.device)
        _check(lib.mfft_sar_quantize(self._ctx, na, nr, _p(raw), _p(h), _p(sc), _stream(raw)))
        return h, sc

    def forward(self, raw_h, pulse_scale, phase):
        import torch
        img = torch.empty_like(raw_h)
        isc = torch.empty(self.params.range_n, dtype=torch.float32, device=raw_h.device)
        _check(lib.mfft_sar_forward(self._h, _p(raw_h), _p(pulse_scale), _p(phase), _p(img), _p(isc),
                                    _stream(raw_h)))
        return img, isc

    def backward_phase(self, raw_h, pulse_scale, phase):
        import torch
        d = torch.empty(self.params.pulses, dtype=torch.float32, device=raw_h.device)
        loss = torch.empty(1, dtype=torch.float64, device=raw_h.device)
        _check(lib.mfft_sar_backward_phase(self._h, _p(raw_h), _p(pulse_scale), _p(phase), _p(d), _p(loss),
                                           _stream(raw_h)))
        return d, loss

    def step(self, raw_h, pulse_scale, phase, out=None):
        """Forward + backward as one CUDA graph (captured once per buffers)."""
        import torch
        if out is None:
            out = (torch.empty_like(raw_h),
                   torch.empty(self.params.range_n, dtype=torch.float32, device=raw_h.device),
                   torch.empty(self.params.pulses, dtype=torch.float32, device=raw_h.device),
                   torch.empty(1, dtype=torch.float64, device=raw_h.device))
        img, isc, d, loss = out
        _check(lib.mfft_sar_step_graph(self._h, _p(raw_h), _p(pulse_scale), _p(phase), _p(img), _p(isc), _p(d),
                                       _p(loss), _stream(raw_h)))
        return out

    @staticmethod
    def to_complex(h, scale, axis_scale):
        """FP16 (.., 2) storage and its scales -> complex64; axis_scale 0 =
        one scale per row (pulse), 1 = per column (range bin)."""
        v = h.float()
        c = v[..., 0] + 1j * v[..., 1]
        return c * (scale[:, None] if axis_scale == 0 else scale[None, :])
