"""Pins the CPU oracle (oracle/) before it is trusted as the checker.

Anchors, in the absence of golden data files in the reference (its tests use
unseeded Float.random):
  * the reference's known-answer tests -- impulse -> all ones
    (Tests/MetalFFTTests/MetalFFTTests.swift:11-23), cosine at bin 100
    (:37-49), the sum of sinusoids at bins 100/200/500 (src/fft_host.swift:409-421),
    DC, the DFT8 matrices and the CT-DIF twiddle table of the tensor-core kernel
    (Tests/MetalFFTTests/DemoComparisonTests.swift:189-233) and "all FFT
    variants agree" (:64-86);
  * numpy's pocketfft, standing in for the reference's comparison path Apple
    vDSP (vDSP_fft_zop, MetalFFTTests.swift:164-188), at the reference's L2
    thresholds (1e-4 package tests, 1e-5 demo validation);
  * the committed golden fixtures of tests/golden/ (make_golden.py).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

SIZES = [64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384]
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def l2(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    den = np.sum(np.abs(b) ** 2)
    num = np.sum(np.abs(a - b) ** 2)
    return float(np.sqrt(num / den) if den > 0 else np.sqrt(num))


def test_fft64_matches_exact_dft():
    for n in [64, 128, 256, 1024]:
        x = O.uniform_c64((n,), seed=n).astype(np.complex128)
        assert l2(O.fft64(x), O.dft(x)) < 1e-14
        assert l2(O.fft64(x, sign=+1), O.dft(x, sign=+1)) < 1e-14


@pytest.mark.parametrize("n", SIZES + [1 << 15, 1 << 20])
def test_fft64_matches_pocketfft(n):
    x = O.normal_c64((2, n), seed=7 + n)
    assert l2(O.truth(x), np.fft.fft(x.astype(np.complex128), axis=-1)) < 1e-13
    assert l2(O.truth(x, inverse=True), np.fft.ifft(x.astype(np.complex128), axis=-1)) < 1e-13


@pytest.mark.parametrize("n", SIZES)
def test_impulse_gives_all_ones(n):
    x = np.zeros((1, n), np.complex64)
    x[0, 0] = 1
    y = O.truth(x)
    assert np.max(np.abs(y - 1.0)) < 1e-12
    yr = O.ref_fft(x)
    assert np.max(np.abs(yr - 1.0)) < 1e-3  # MetalFFTTests.swift:19-20 accuracy


def test_dc_gives_n_at_bin_zero():
    n = 4096
    x = np.ones((1, n), np.complex64)
    y = O.truth(x)[0]
    assert abs(y[0] - n) < 1e-9 and np.max(np.abs(y[1:])) < 1e-9


def test_cosine_peak_bin_100():
    n = 1024
    k = np.arange(n)
    x = np.cos(2 * np.pi * 100 * k / n).astype(np.complex64)[None]
    mags = np.abs(O.truth(x)[0, : n // 2]) ** 2
    assert int(np.argmax(mags)) == 100
    assert int(np.argmax(np.abs(O.ref_fft(x)[0, : n // 2]))) == 100


def test_sum_of_sinusoids_bins():
    # x[k] = cos(100 t) + 0.5 cos(200 t) + 0.3 sin(500 t), t = 2 pi k / N
    n = 4096
    t = 2 * np.pi * np.arange(n) / n
    x = (np.cos(100 * t) + 0.5 * np.cos(200 * t) + 0.3 * np.sin(500 * t)).astype(np.complex64)
    y = O.truth(x[None])[0]
    assert abs(y[100] - n / 2) < 1e-2 and abs(y[n - 100] - n / 2) < 1e-2
    assert abs(y[200] - n / 4) < 1e-2
    assert abs(y[500] - (-0.3j * n / 2)) < 1e-2 and abs(y[n - 500] - (0.3j * n / 2)) < 1e-2
    others = np.delete(np.abs(y), [100, n - 100, 200, n - 200, 500, n - 500])
    assert others.max() < 1e-2


@pytest.mark.parametrize("n", SIZES + [1 << 15, 1 << 16, 1 << 18, 1 << 20])
def test_reference_fp32_path_vs_fp64(n):
    """The FP32 restatement of the reference path is within the reference's
    demo threshold (L2 < 1e-5, src/fft_host.swift:467) of FP64, forward and
    inverse, for every size including the four-step ones."""
    batch = 2 if n <= 16384 else 1
    x = O.uniform_c64((batch, n), seed=11 + n)
    assert O.rel_rms(O.ref_fft(x), O.truth(x)) < 1e-5
    assert O.rel_rms(O.ref_fft(x, inverse=True), O.truth(x, inverse=True)) < 1e-5


def test_reference_fourstep_splits():
    # MetalContext.swift:57-66
    assert O.ref_fourstep_split(8192) == (64, 128)
    assert O.ref_fourstep_split(16384) == (128, 128)
    assert O.ref_fourstep_split(1 << 20) == (1024, 1024)


def test_batch_matches_single():
    n = 512
    x = O.uniform_c64((2, n), seed=3)
    yb = O.ref_fft(x)
    for i in range(2):
        assert l2(yb[i], O.ref_fft(x[i : i + 1])[0]) < 1e-6


# ---- DFT8 matrices and the CT-DIF algorithm of src/fft_4096_ct_mma.metal -----

S2 = np.sqrt(0.5)


def _dft8_table():
    """DFT_8 real/imag tables as the reference test builds them
    (DemoComparisonTests.swift:194-213): entries in {0, +-1, +-sqrt(1/2)}."""
    codes_re = [
        [1, 1, 1, 1, 1, 1, 1, 1], [1, 2, 0, -2, -1, -2, 0, 2], [1, 0, -1, 0, 1, 0, -1, 0],
        [1, -2, 0, 2, -1, 2, 0, -2], [1, -1, 1, -1, 1, -1, 1, -1], [1, -2, 0, 2, -1, 2, 0, -2],
        [1, 0, -1, 0, 1, 0, -1, 0], [1, 2, 0, -2, -1, -2, 0, 2]]
    codes_im = [
        [0] * 8, [0, -2, -1, -2, 0, 2, 1, 2], [0, -1, 0, 1, 0, -1, 0, 1],
        [0, -2, 1, -2, 0, 2, -1, 2], [0] * 8, [0, 2, -1, 2, 0, -2, 1, -2],
        [0, 1, 0, -1, 0, 1, 0, -1], [0, 2, 1, 2, 0, -2, -1, -2]]

    def val(c):
        return {0: 0.0, 1: 1.0, -1: -1.0, 2: S2, -2: -S2}[c]
    re = np.array([[val(c) for c in row] for row in codes_re])
    im = np.array([[val(c) for c in row] for row in codes_im])
    return re + 1j * im


def test_dft8_matrix_entries():
    F = _dft8_table()
    for j in range(8):
        e = np.zeros(8, np.complex128)
        e[j] = 1
        assert np.max(np.abs(O.dft(e) - F[:, j])) < 1e-15


def _ct_twiddles(n=4096):
    """Twiddle table of the CT-DIF stages (DemoComparisonTests.swift:215-233):
    stride S, group G: element i gets exp(-2 pi i r k / G), r = (i % G) / S,
    k = (i % G) % S."""
    tab = np.ones((3, n), np.complex128)
    for st, (S, G) in enumerate([(512, 4096), (64, 512), (8, 64)]):
        i = np.arange(n)
        r = (i % G) // S
        k = (i % G) % S
        tab[st] = np.exp(-2j * np.pi * r * k / G)
    return tab


def _ct_dif_4096(x):
    """Restatement of fft_4096_ct_mma's algorithm (src/fft_4096_ct_mma.metal
    :88-206): three radix-8 DIF stages as DFT8 matmuls + table twiddles, a
    scalar radix-8 stage, base-8 digit reversal on store."""
    F = _dft8_table()
    tw = _ct_twiddles()
    buf = np.asarray(x, np.complex128).copy()
    for st, S in enumerate([512, 64, 8]):
        G = 8 * S
        b = buf.reshape(4096 // G, 8, S)
        y = np.einsum("rn,gnk->grk", F, b).reshape(4096)
        buf = y * tw[st]
    y = (buf.reshape(512, 8) @ F.T).reshape(4096)
    idx = np.arange(4096)
    rev = ((idx & 7) << 9) | (((idx >> 3) & 7) << 6) | (((idx >> 6) & 7) << 3) | ((idx >> 9) & 7)
    out = np.empty_like(y)
    out[rev] = y
    return out


def test_ct_dif_variant_agrees_with_oracle():
    x = O.uniform_c64((1, 4096), seed=5)
    assert l2(_ct_dif_4096(x[0]), O.truth(x)[0]) < 1e-13
    # twiddle-table spot values: stage 0 entry for r=1, k=1 is exp(-2 pi i / 4096)
    tab = _ct_twiddles()
    assert abs(tab[0, 512 + 1] - np.exp(-2j * np.pi / 4096)) < 1e-15
    assert np.all(tab[:, 0] == 1)


# ---- golden fixtures --------------------------------------------------------

def _golden(name):
    return np.load(os.path.join(GOLDEN, name))


def test_golden_fft_fixtures():
    # fixtures from pocketfft (tests/golden/make_golden.py), not from the oracle
    z = _golden("fft_golden.npz")
    for n in [64, 512, 4096]:
        x, X, Xi = z["x_%d" % n], z["X_%d" % n], z["Xi_%d" % n]
        assert l2(O.truth(x), X) < 1e-13
        assert l2(O.truth(x, inverse=True), Xi) < 1e-13
        assert l2(O.fft64(x), X) < 1e-13
        assert O.rel_rms(O.ref_fft(x), X) < 1e-6          # the FP32 restatement
        assert O.rel_rms(O.ref_fft(x, inverse=True), Xi) < 1e-6


def test_golden_convolver_fixtures():
    """The oracle's FP64 overlap-add, its FP32 restatement of the reference's
    loop and its analytic adjoint against the transliterated reference loop
    (Convolve.swift:36-76) on the reference's edge cases: an empty signal, a
    signal shorter than one hop, K = 1, a signal ending on a hop boundary,
    hop 2."""
    z = _golden("conv_golden.npz")
    for name in z["cases"]:
        x, h, y, t = z[name + "_x"], z[name + "_h"], z[name + "_y"], z[name + "_t"]
        fft = int(z[name + "_fft"])
        assert y.shape == (len(x) + len(h) - 1,)
        y64 = O.conv64(x, h, fft)
        assert y64.shape == y.shape, name
        scale = max(np.max(np.abs(y)), 1e-30)
        assert np.max(np.abs(y64 - y)) <= 1e-12 * scale, name
        y32 = O.ref_conv(x, h, fft)
        assert y32.shape == y.shape, name
        assert np.max(np.abs(y32 - y)) <= 2e-6 * scale, name
        if len(x) == 0:
            assert not y64.any() and not y32.any()
            continue
        dx, dh = O.conv_adjoint64(x, h, (y - t))
        assert np.max(np.abs(dx - z[name + "_dx"])) <= 1e-11 * np.max(np.abs(z[name + "_dx"])), name
        assert np.max(np.abs(dh - z[name + "_dh"])) <= 1e-11 * np.max(np.abs(z[name + "_dh"])), name


def test_golden_correlator_fixtures():
    """corr64 / ref_corr against the transliterated Correlator.cross
    (Correlate.swift:27-61): zero padding, truncation of inputs longer than
    fftSize, an empty input, and auto()."""
    z = _golden("corr_golden.npz")
    for name in z["cases"]:
        a, b, r = z[name + "_a"], z[name + "_b"], z[name + "_r"]
        fft = int(z[name + "_fft"])
        scale = max(np.max(np.abs(r)), 1e-30)
        assert np.max(np.abs(O.corr64(a, b, fft) - r)) <= 1e-12 * scale, name
        assert np.max(np.abs(O.ref_corr(a, b, fft) - r)) <= 2e-6 * max(scale, np.sum(a * a)), name


def test_golden_window_and_analyzer_fixtures():
    """The flat-top and Kaiser coefficients and FFTAnalyzer.analyze (window x
    samples in FP32, FFT) against the transliterated reference
    (Window.swift:51-75,100-110, FFTAnalyzer.swift:93-116)."""
    z = _golden("analyzer_golden.npz")
    n = len(z["w_rect"])
    assert np.max(np.abs(O.window(3, n) - z["w_flattop"])) < 1e-6
    assert np.max(np.abs(O.window(4, n, 6.0) - z["w_kaiser6"])) < 1e-9
    assert np.max(np.abs(O.window(4, n, 9.5) - z["w_kaiser9"])) < 1e-9
    assert np.all(O.window(5, n) == 1.0)
    s = z["samples"]
    for key, kind, beta in [("flattop", 3, 6.0), ("kaiser6", 4, 6.0), ("kaiser9", 4, 9.5), ("rect", 5, 6.0)]:
        w = np.asarray(O.window(kind, n, beta), np.float32)
        for tag, off in [("X0_", 0), ("X1_", n + 17)]:
            win = (s[off:off + n] * w).astype(np.float32)
            assert l2(O.fft64(win.astype(np.complex128)[None])[0], z[tag + key]) < 1e-6, (key, tag)


# ---- convolver / correlator --------------------------------------------------

def test_conv64_matches_direct():
    rng = np.random.default_rng(1)
    x = rng.standard_normal(300)
    h = rng.standard_normal(31)
    y = O.conv64(x, h, 64)
    assert np.max(np.abs(y - np.convolve(x, h))) < 1e-12


def test_ref_conv_matches_fp64():
    rng = np.random.default_rng(2)
    x = rng.standard_normal(8192 * 2).astype(np.float32)
    h = rng.standard_normal(128).astype(np.float32)
    y = O.ref_conv(x, h, 4096)
    y64 = O.conv64(x, h, 4096)
    assert np.linalg.norm(y - y64) / np.linalg.norm(y64) < 1e-5


def test_delta_kernel_is_identity():
    # FusedConvolverTests.swift:11-22
    h = np.zeros(64, np.float32)
    h[0] = 1
    x = np.random.default_rng(3).uniform(-1, 1, 4096 - 63).astype(np.float32)
    y = O.ref_conv(x, h, 4096)
    assert np.linalg.norm(y[: len(x)] - x) / np.linalg.norm(x) < 1e-4


def test_conv_adjoint_vs_central_differences():
    rng = np.random.default_rng(4)
    nx, K = 60, 9
    x = rng.standard_normal(nx)
    h = rng.standard_normal(K)
    t = rng.standard_normal(nx + K - 1)

    def loss(x_, h_):
        return 0.5 * np.sum((np.convolve(x_, h_) - t) ** 2)

    g = np.convolve(x, h) - t
    dx, dh = O.conv_adjoint64(x, h, g)
    eps = 1e-6
    for i in range(nx):
        e = np.zeros(nx)
        e[i] = eps
        fd = (loss(x + e, h) - loss(x - e, h)) / (2 * eps)
        assert abs(fd - dx[i]) < 1e-5 * max(1.0, abs(fd))
    for k in range(K):
        e = np.zeros(K)
        e[k] = eps
        fd = (loss(x, h + e) - loss(x, h - e)) / (2 * eps)
        assert abs(fd - dh[k]) < 1e-5 * max(1.0, abs(fd))


def test_corr_matches_definition():
    rng = np.random.default_rng(5)
    n = 256
    a = rng.standard_normal(200)
    b = rng.standard_normal(300)  # truncated to n
    r = O.corr64(a, b, n)
    ap = np.zeros(n)
    ap[:200] = a
    bp = b[:n]
    # The code computes IFFT(A * conj(B)) (Correlate.swift:41-45), i.e.
    # R[m] = sum_n a[n+m] b[n]; its doc comment's sum_n a[n] b[n+m] is the
    # mirrored lag.  Parity follows the code.
    direct = np.array([np.sum(np.roll(ap, -m) * bp) for m in range(n)])
    assert np.max(np.abs(r - direct)) < 1e-10
    assert np.max(np.abs(O.ref_corr(a, b, n) - r)) < 1e-4 * np.max(np.abs(r))


def test_autocorr_peak_is_energy():
    x = np.random.default_rng(6).standard_normal(100)
    r = O.corr64(x, x, 256)
    assert abs(r[0] - np.sum(x * x)) < 1e-10
    assert np.argmax(r) == 0


def test_windows():
    w = O.window(0, 1024)
    assert w[0] == 0.0  # MetalFFTTests.swift:69-73
    assert abs(w[512] - 0.8165 * 2) < 1e-12
    hm = O.window(1, 8)
    assert abs(hm[0] - 0.08) < 1e-12
    assert np.all(O.window(5, 16) == 1.0)
    k = O.window(4, 33, 6.0)
    assert abs(k[16] - 1.0) < 1e-12 and abs(k[0] - k[32]) < 1e-12


# ---- STFT / Welch / coherence oracle (DSP/STFT.swift, DSP/PSD.swift) --------

def test_stft_oracle_matches_per_frame_pocketfft():
    rng = np.random.default_rng(5)
    x = rng.standard_normal(3000)
    for fft, hop, kind in [(256, 128, 0), (256, 100, 4), (64, 64, 5)]:
        w = O.window(kind, fft)
        S = O.stft64(x, fft, hop, w)
        frames = (len(x) - fft) // hop + 1  # STFT.swift:58-61
        assert S.shape == (frames, fft) == (O.stft_frames(len(x), fft, hop), fft)
        ref = np.fft.fft(np.stack([w * x[f * hop:f * hop + fft] for f in range(frames)]), axis=1)
        assert np.abs(S - ref).max() < 1e-11 * np.abs(ref).max()
    assert O.stft_frames(100, 256, 64) == 0


def test_welch_oracle_known_answers():
    # PSD.swift:53-56 normalisation, and a tone at an exact bin of a
    # rectangular window: all power in bins b and N-b, sum = A^2 N / (2 fs)
    fft, hop, fs, b, amp = 256, 128, 1000.0, 19, 1.5
    n = 256 * 20
    t = np.arange(n)
    x = amp * np.cos(2 * np.pi * b * t / fft)
    w = O.window(5, fft)
    P = O.welch64(x, fft, hop, w, fs)
    assert np.argmax(P[:fft // 2]) == b
    others = np.delete(P, [b, fft - b])
    assert others.max() < 1e-20
    assert abs(P[b] - (amp / 2) ** 2 * fft / fs) < 1e-9 * P[b]
    # no frame: zeros
    assert not O.welch64(x[:100], fft, hop, w, fs).any()


def test_coherence_oracle_known_answers():
    rng = np.random.default_rng(6)
    x = rng.standard_normal(8192)
    y = rng.standard_normal(8192)
    w = O.window(0, 256)
    assert np.allclose(O.coherence64(x, 3.0 * x, 256, 128, w), 1.0, atol=1e-12)
    c = O.coherence64(x, y, 256, 128, w)
    assert 0.0 <= c.min() and c.max() < 0.5 and c.mean() < 0.05  # independent noise, 63 frames
    assert not O.coherence64(x[:100], y, 256, 128, w).any()


def test_cross_spectral_oracle_known_answers():
    # CrossSpectral.swift:56-152 / fft_cross_spectral.metal:29-63 restated:
    # power = mean |X_c|^2 (the Welch PSD without its normalisation), cross =
    # mean X_i conj(X_j), coherence = mean of per-frame |S|^2 / (p_i p_j) = 1
    # wherever both channels have power, whatever the channels are
    rng = np.random.default_rng(8)
    x = rng.standard_normal((3, 4096))
    fft, hop, fs = 256, 128, 1000.0
    w = O.window(0, fft)
    pw, cr, ch = O.cross_spectral64(x, fft, hop, w)
    assert pw.shape == (3, fft) and cr.shape == (3, fft) and ch.shape == (3, fft)
    wss = float(np.sum(w * w))
    for c in range(3):
        assert np.allclose(pw[c], O.welch64(x[c], fft, hop, w, fs) * wss * fs, rtol=1e-12)
    S = [O.stft64(x[c], fft, hop, w) for c in range(3)]
    for q, (i, j) in enumerate([(0, 1), (0, 2), (1, 2)]):
        assert np.allclose(cr[q], np.mean(S[i] * np.conj(S[j]), axis=0), rtol=1e-12, atol=1e-9)
    assert np.allclose(ch, 1.0, atol=1e-12)
    # the Welch estimate from these averages is PSD.coherence
    assert np.allclose(np.abs(cr[0]) ** 2 / (pw[0] * pw[1]), O.coherence64(x[0], x[1], fft, hop, w), atol=1e-12)
    # zero channels: per-frame 0 / max(0, 1e-30) = 0; too short: all zeros
    z = O.cross_spectral64(np.zeros((2, 1024)), fft, hop, w)
    assert not z[0].any() and not z[1].any() and not z[2].any()
    s = O.cross_spectral64(x[:, :100], fft, hop, w)
    assert not s[0].any() and not s[2].any()
    one = O.cross_spectral64(x[:1], fft, hop, w)
    assert one[1].shape == (0, fft) and one[2].shape == (0, fft)


def test_cross_spectral_pair_index():
    # CrossSpectral.swift:29-37 and CrossSpectralTests.swift:102-118
    from metalfft_b200 import CrossSpectralResult
    r = CrossSpectralResult(4, 1024, None, None, None)
    assert [r.pair_index(i, j) for i, j in [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]] == list(range(6))
    assert r.pair_count == 6
    r16 = CrossSpectralResult(16, 64, None, None, None)
    flat = [(i, j) for i in range(16) for j in range(i + 1, 16)]
    assert [r16.pair_index(i, j) for i, j in flat] == list(range(120))
    with pytest.raises(ValueError):
        r.pair_index(2, 1)
