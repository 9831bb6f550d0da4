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


RC_FP16, RC_FP32 = 0, 1


class SARPipeline:
    """Range compression -> corner turn -> azimuth FFT on device tensors.
    intermediate: RC_FP16 (default, FP16 with per-pulse scales between the
    passes) or RC_FP32 (the precision the phase adjoint needs for ~1e-5)."""

    def __init__(self, params, chirp=None, context=None):
        self.params = params
        c = np.ascontiguousarray(chirp if chirp is not None else params.chirp_reference(), np.complex64)
        self._ctx = context or shared_context()
        h = ctypes.c_void_p()
        _check(lib.mfft_sar_create(self._ctx, ctypes.byref(params), c.ctypes.data, ctypes.byref(h)))
        self._h = h

    def set_intermediate(self, precision):
        """RC_FP16 or RC_FP32 for later forward / backward_phase / step calls."""
        _check(lib.mfft_sar_set_intermediate(self._h, int(precision)))

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

    def focus(self, image_h, image_scale, reference_signs=False):
        """Focused image (FP16, one scale per range column) from the
        range-Doppler image of forward(): RCMC, azimuth matched filter and
        inverse azimuth FFT (rda_kernels.metal:103-240).  reference_signs
        reproduces the reference's RCMC direction and filter sign."""
        import torch
        out = torch.empty_like(image_h)
        osc = torch.empty(self.params.range_n, dtype=torch.float32, device=image_h.device)
        _check(lib.mfft_sar_focus(self._h, _p(image_h), _p(image_scale), _p(out), _p(osc),
                                  1 if reference_signs else 0, _stream(image_h)))
        return out, osc

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


def expected_bins(params, target):
    """(range bin, azimuth bin) where a point target focuses
    (src/radar/sar_simulator.swift:118-119)."""
    c = 299792458.0
    tau0 = 2.0 * params.center_range / c - (params.range_n // 2) / params.sample_rate
    rg = int((2.0 * target.range_m / c - tau0) * params.sample_rate)
    az = int((target.azimuth_m / params.velocity + (params.pulses // 2) / params.prf) * params.prf)
    return rg, az


def point_target_metrics(power, expected_rg, expected_az, radius=20):
    """RadarMetrics.measureTarget (src/radar/radar_metrics.swift:57-268) on a
    |I|^2 image (azimuth x range): peak search, range / azimuth cuts through
    the peak, PSLR and ISLR against a -20 dB mainlobe, -3 dB widths, and SNR
    of the peak over the two 64 x 64 corners."""
    import numpy as np
    m = np.asarray(power, dtype=np.float64)
    na, nr = m.shape
    a0, a1 = max(0, expected_az - radius), min(na - 1, expected_az + radius)
    r0, r1 = max(0, expected_rg - radius), min(nr - 1, expected_rg + radius)
    win = m[a0:a1 + 1, r0:r1 + 1]
    ia, ir = np.unravel_index(int(np.argmax(win)), win.shape)
    pa, pr = a0 + int(ia), r0 + int(ir)
    peak = m[pa, pr]

    def cut_metrics(cut, pk):
        n = len(cut)
        pv = cut[pk]
        if pv <= 0:
            return 0.0, 0.0, float(n)
        db = lambda v: 10 * np.log10(v / pv) if v > 0 else -100.0  # noqa: E731
        left = pk
        for i in range(pk - 1, -1, -1):
            if db(cut[i]) < -20.0:
                left = i + 1
                break
            if i == 0:
                left = 0
        right = pk
        for i in range(pk + 1, n):
            if db(cut[i]) < -20.0:
                right = i - 1
                break
            if i == n - 1:
                right = n - 1
        main = float(cut[left:right + 1].sum())
        half = min(n // 4, 200)
        wl, wr = max(0, pk - half), min(n - 1, pk + half)
        side = [cut[i] for i in range(wl, wr + 1) if i < left or i > right]
        side_e = float(np.sum(side)) if side else 0.0
        side_max = float(np.max(side)) if side else 0.0
        pslr = 10 * np.log10(side_max / pv) if side_max > 0 else -60.0
        islr = 10 * np.log10(side_e / main) if side_e > 0 and main > 0 else -60.0
        thr = pv * 0.5
        l3 = float(pk)
        for i in range(pk, max(0, pk - half) - 1, -1):
            if cut[i] < thr:
                l3 = i + (thr - cut[i]) / (cut[i + 1] - cut[i]) if i + 1 < n and cut[i + 1] > thr else float(i)
                break
        r3 = float(pk)
        for i in range(pk, min(n, pk + half)):
            if cut[i] < thr:
                r3 = i - (thr - cut[i]) / (cut[i - 1] - cut[i]) if i > 0 and cut[i - 1] > thr else float(i)
                break
        return pslr, islr, r3 - l3

    pslr_r, islr_r, res_r = cut_metrics(m[pa, :], pr)
    pslr_a, islr_a, res_a = cut_metrics(m[:, pr], pa)
    cs = 64
    noise = np.concatenate([m[:cs, :cs].ravel(), m[na - cs:, nr - cs:].ravel()]).mean()
    snr = 10 * np.log10(peak / noise) if noise > 0 else 60.0
    return {"range_bin": pr, "azimuth_bin": pa, "peak": float(peak), "pslr_range": pslr_r,
            "pslr_azimuth": pslr_a, "islr_range": islr_r, "islr_azimuth": islr_a, "snr": snr,
            "res3db_range": res_r, "res3db_azimuth": res_a}
