"""PSD.crossSpectral (DSP/CrossSpectral.swift:56-152) on the GPU through
libmfft's C ABI, against the FP64 oracle, plus the reference's own checks
(Tests/MetalFFTTests/CrossSpectralTests.swift)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


def _w(kind, fft, beta=6.0):
    return O.window(kind, fft, beta).astype(np.float32).astype(np.float64)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


# channel counts cover every pair split (1, 2, 4 and 8 warp groups); the long
# cases run through several L2-sized chunks, odd frame counts included
@pytest.mark.parametrize("C,fft,hop,kind,n", [
    (1, 256, 128, 0, 4096), (2, 64, 32, 1, 5000), (3, 1024, 512, 0, 1 << 14), (6, 512, 200, 4, 30000),
    (7, 1024, 512, 0, 1 << 15), (8, 4096, 1024, 2, 1 << 16), (9, 256, 128, 0, 20000), (12, 2048, 1024, 0, 1 << 15),
    (16, 1024, 512, 0, 512 * 1201 + 512), (16, 16384, 8192, 0, 8192 * 33), (5, 64, 64, 0, 64 * 2100 + 7),
    (4, 512, 256, 1, 1 << 14)])
def test_cross_spectral_matches_fp64(M, C, fft, hop, kind, n):
    rng = np.random.default_rng(C * 1000 + fft)
    base = rng.standard_normal(n)
    x = np.stack([0.6 * base + rng.standard_normal(n) for _ in range(C)]).astype(np.float32)
    r = M.PSD.cross_spectral(x, fft, hop, 48000.0, M.WindowType(kind, 6.0))
    pw, cr, ch = O.cross_spectral64(x.astype(np.float64), fft, hop, _w(kind, fft))
    P = C * (C - 1) // 2
    assert r.channels == C and r.fft_size == fft and r.pair_count == P
    assert r.power.shape == (C, fft) and r.cross_spectra.shape == (P, fft) and r.coherence.shape == (P, fft)
    assert float(np.max(np.abs(r.power - pw)) / pw.max()) < 3e-6
    if P:
        assert _rel(r.cross_spectra, cr) < 1e-5
        assert float(np.max(np.abs(r.coherence - ch))) < 1e-5


def test_identical_channels_have_unit_coherence(M):
    # CrossSpectralTests.swift:66-87
    x = np.random.default_rng(3).uniform(-1, 1, 1024 * 4).astype(np.float32)
    r = M.PSD.cross_spectral([x, x, x], 1024, 512, 44100.0)
    assert r.channels == 3 and r.pair_count == 3
    assert np.allclose(r.coherence[:, 1:], 1.0, atol=1e-4)
    rw = M.PSD.cross_spectral([x, x, x], 1024, 512, 44100.0, coherence_mode=M.COHERENCE_WELCH)
    assert np.allclose(rw.coherence[:, 1:], 1.0, atol=1e-4)


def test_single_channel_power_is_scaled_welch(M):
    # CrossSpectralTests.swift:89-100, 120-145: no pairs; the power is the
    # Welch PSD without its 1 / (sum w^2 * sample rate) normalisation
    x = np.random.default_rng(4).uniform(-1, 1, 1024 * 8).astype(np.float32)
    r = M.PSD.cross_spectral([x], 1024, 512, 44100.0)
    assert r.pair_count == 0 and r.power.shape == (1, 1024)
    assert r.cross_spectra.shape == (0, 1024) and r.coherence.shape == (0, 1024)
    psd = M.PSD.welch(x, 1024, 512, 44100.0)
    wss = float(np.sum(_w(0, 1024) ** 2))
    assert float(np.max(np.abs(r.power[0] - psd * wss * 44100.0)) / r.power.max()) < 3e-6


def test_pair_index_ordering(M):
    # CrossSpectralTests.swift:102-118
    x = np.random.default_rng(5).uniform(-1, 1, 1024 * 2).astype(np.float32)
    r = M.PSD.cross_spectral([x] * 4, 1024, 512, 44100.0)
    assert [r.pair_index(i, j) for i, j in [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]] == list(range(6))
    assert r.pair_count == 6


def test_coherence_bounds_and_welch_mode(M):
    # CrossSpectralTests.swift:147-172, and the Welch estimate against
    # PSD.coherence of every pair
    rng = np.random.default_rng(6)
    s1 = rng.uniform(-1, 1, 1024 * 4).astype(np.float32)
    s2 = (0.5 * rng.uniform(-1, 1, 1024 * 4) + 0.5 * s1).astype(np.float32)
    s3 = rng.uniform(-1, 1, 1024 * 4).astype(np.float32)
    r = M.PSD.cross_spectral([s1, s2], 1024, 512, 44100.0)
    assert r.coherence.min() >= -1e-6 and r.coherence.max() <= 1 + 1e-6
    rw = M.PSD.cross_spectral([s1, s2, s3], 1024, 512, 44100.0, coherence_mode=M.COHERENCE_WELCH)
    assert rw.coherence.min() >= -1e-6 and rw.coherence.max() <= 1 + 1e-6
    for (i, j), a, b in [((0, 1), s1, s2), ((0, 2), s1, s3), ((1, 2), s2, s3)]:
        ref = M.PSD.coherence(a, b, 1024, 512)
        assert float(np.max(np.abs(rw.coherence[rw.pair_index(i, j)] - ref))) < 1e-5
    # Welch coherence from the FP64 oracle's averaged outputs
    pw, cr, _ = O.cross_spectral64(np.stack([s1, s2, s3]).astype(np.float64), 1024, 512, _w(0, 1024))
    den = pw[[0, 0, 1]] * pw[[1, 2, 2]]
    assert float(np.max(np.abs(rw.coherence - np.abs(cr) ** 2 / den))) < 1e-5


def test_zero_frames_and_errors(M):
    short = np.ones((2, 100), np.float32)
    r = M.PSD.cross_spectral(short, 256, 128)
    assert not r.power.any() and not r.cross_spectra.any() and not r.coherence.any()
    x = np.zeros(2048, np.float32)
    with pytest.raises(M.FFTError) as e:
        M.PSD.cross_spectral([x] * 17, 1024, 512)
    assert e.value.case == "invalidArgument"
    with pytest.raises(M.FFTError):
        M.PSD.cross_spectral([], 1024, 512)
    with pytest.raises(M.FFTError):
        M.PSD.cross_spectral([x, x[:-1]], 1024, 512)
    with pytest.raises(M.FFTError):
        M.PSD.cross_spectral([x, x], 1024, 512, coherence_mode=2)
    with pytest.raises(M.FFTError) as e:
        M.PSD.cross_spectral([x, x], 1000, 512)
    assert e.value.case == "unsupportedFFTSize"
    # all-zero channels: power 0, per-frame coherence 0 / max(0, 1e-30) = 0
    z = M.PSD.cross_spectral([x, x], 1024, 512)
    assert not z.power.any() and not z.coherence.any()


def test_device_tensors_match_host(M):
    import torch
    rng = np.random.default_rng(7)
    x = rng.standard_normal((5, 1 << 16)).astype(np.float32)
    est = M.SpectralEstimator(2048, 1024, M.WindowType(1))
    hp, hc, hh = est.cross_spectral(x)
    dp, dc, dh = est.cross_spectral(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(hp, dp.cpu().numpy())
    assert np.array_equal(hc, dc.cpu().numpy())
    assert np.array_equal(hh, dh.cpu().numpy())
    # repeated calls on one handle are deterministic (fixed-order sums)
    dp2, dc2, dh2 = est.cross_spectral(torch.from_numpy(x).cuda())
    assert torch.equal(dp, dp2) and torch.equal(dc, dc2) and torch.equal(dh, dh2)


@pytest.mark.parametrize("C,fft", [(2, 256), (4, 1024), (8, 1024)])
def test_welch_mode_compile_time_channel_counts(M, C, fft):
    # 2, 4 and 8 channels take the kernel whose channel count is a template
    # constant; the Welch estimate |mean S_ij|^2 / (mean p_i mean p_j) against
    # the FP64 oracle's averaged powers and cross-spectra
    rng = np.random.default_rng(C + fft)
    n = fft * 40 + 3
    base = rng.standard_normal(n)
    x = np.stack([0.5 * base + rng.standard_normal(n) for _ in range(C)]).astype(np.float32)
    rw = M.PSD.cross_spectral(x, fft, fft // 2, 48000.0, coherence_mode=M.COHERENCE_WELCH)
    pw, cr, _ = O.cross_spectral64(x.astype(np.float64), fft, fft // 2, _w(0, fft))
    assert float(np.max(np.abs(rw.power - pw)) / pw.max()) < 3e-6
    assert _rel(rw.cross_spectra, cr) < 1e-5
    ii, jj = np.triu_indices(C, 1)
    den = pw[ii] * pw[jj]
    assert float(np.max(np.abs(rw.coherence - np.abs(cr) ** 2 / den))) < 1e-5
