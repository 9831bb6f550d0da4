"""STFT, Welch PSD and coherence (DSP/STFT.swift, DSP/PSD.swift) on the GPU
through libmfft's C ABI, against the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("fft,hop,kind,n", [
    (64, 32, 0, 4096), (256, 100, 4, 20000), (1024, 512, 1, 1 << 16), (4096, 1024, 2, 1 << 18),
    (16384, 4096, 0, 1 << 18), (512, 512, 5, 512 * 7 + 11)])
def test_stft_matches_fp64(M, fft, hop, kind, n):
    x = np.random.default_rng(fft + hop).standard_normal(n).astype(np.float32)
    wt = M.WindowType(kind, 6.0)
    st = M.STFT(fft, hop, wt, sample_rate=48000.0)
    fr = st.analyze(x)
    w = O.window(kind, fft, 6.0)
    ref = O.stft64(x.astype(np.float64), fft, hop, w.astype(np.float32).astype(np.float64))
    assert len(fr) == st.frame_count(n) == O.stft_frames(n, fft, hop)
    assert _rel(fr.complex, ref) < 2e-6
    pref = np.abs(ref) ** 2
    assert float(np.linalg.norm(fr.magnitudes - pref) / np.linalg.norm(pref)) < 4e-6


def test_stft_odd_and_zero_frame_counts(M):
    st = M.STFT(256, 128)
    x = np.random.default_rng(1).standard_normal(256 + 128 * 4).astype(np.float32)  # 5 frames
    fr = st.analyze(x)
    assert len(fr) == 5
    ref = O.stft64(x.astype(np.float64), 256, 128, O.window(0, 256).astype(np.float32).astype(np.float64))
    assert _rel(fr.complex[-1], ref[-1]) < 2e-6  # the unpaired last frame
    assert len(st.analyze(np.zeros(100, np.float32))) == 0
    db = fr.magnitudes_db  # Spectrum.toDecibels: 20 log10(|X|^2), floor -120
    assert db.min() >= -120.0
    assert np.allclose(db, np.maximum(20 * np.log10(np.maximum(fr.magnitudes, 1e-300)), -120), atol=1e-3)


@pytest.mark.parametrize("fft,hop,kind,n", [
    (64, 32, 0, 10000), (256, 128, 1, 1 << 18), (4096, 2048, 0, 1 << 20), (8192, 2048, 4, 1 << 20),
    (16384, 8192, 0, 1 << 20),
    (1024, 512, 0, 1024),                # one frame: its line's imaginary input is zero
    (2048, 1000, 3, 2048 + 2 * 1000)])   # three frames: the last pair holds one
def test_welch_matches_fp64(M, fft, hop, kind, n):
    x = np.random.default_rng(n + fft).standard_normal(n).astype(np.float32)
    wt = M.WindowType(kind, 6.0)
    P = M.PSD.welch(x, fft, hop, 44100.0, wt)
    w = O.window(kind, fft, 6.0).astype(np.float32).astype(np.float64)
    ref = O.welch64(x.astype(np.float64), fft, hop, w, 44100.0)
    assert float(np.max(np.abs(P - ref) / ref.max())) < 2e-6
    assert float(np.linalg.norm(P - ref) / np.linalg.norm(ref)) < 2e-6


@pytest.mark.parametrize("fft,hop", [(256, 128), (4096, 1024), (8192, 4096), (16384, 4096)])
def test_coherence_matches_fp64(M, fft, hop):
    rng = np.random.default_rng(fft)
    n = 1 << 19
    s = rng.standard_normal(n)
    a = (s + 0.5 * rng.standard_normal(n)).astype(np.float32)
    b = (np.convolve(s, [0.5, 0.3, -0.2], mode="same") + 0.5 * rng.standard_normal(n)).astype(np.float32)
    C = M.PSD.coherence(a, b[: n - 5], fft, hop)  # min(na, nb) samples, PSD.swift:98
    w = O.window(0, fft).astype(np.float32).astype(np.float64)
    ref = O.coherence64(a.astype(np.float64), b[: n - 5].astype(np.float64), fft, hop, w)
    assert float(np.abs(C - ref).max()) < 5e-5
    assert np.allclose(M.PSD.coherence(a, a, fft, hop), 1.0, atol=1e-5)


def test_device_tensors_match_host(M):
    import torch
    x = np.random.default_rng(3).standard_normal(1 << 18).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    st = M.STFT(1024, 256)
    spec, power = st.analyze(xd)
    fr = st.analyze(x)
    assert np.array_equal(spec.cpu().numpy(), fr.complex) and np.array_equal(power.cpu().numpy(), fr.magnitudes)
    est = M.SpectralEstimator(1024, 256, None, None)
    p_dev = est.welch(xd, 8000.0).cpu().numpy()
    assert np.array_equal(p_dev, est.welch(x, 8000.0))
    assert np.array_equal(p_dev, M.PSD.welch(x, 1024, 256, 8000.0))


def test_spectral_errors(M):
    for bad in (100, 32768, 32):
        with pytest.raises(M.FFTError) as e:
            M.STFT(bad, 16)
        assert e.value.case == "unsupportedFFTSize"
    with pytest.raises(M.FFTError) as e:
        M.STFT(256, 0)
    assert e.value.case == "invalidArgument"
    assert not M.PSD.welch(np.zeros(10, np.float32), 256, 128, 1.0).any()
    assert not M.PSD.coherence(np.zeros(10, np.float32), np.zeros(300, np.float32), 256, 128).any()
