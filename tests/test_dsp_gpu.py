"""Parity of the fused Convolver / FusedConvolver (and its adjoint), the
Correlator and FFTAnalyzer with the FP64 oracle, following the reference's
FusedConvolverTests.swift and the Correlate/FFTAnalyzer semantics."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_delta_filter_is_identity(M):
    # FusedConvolverTests.swift:11-22
    delta = np.zeros(64, np.float32)
    delta[0] = 1
    conv = M.FusedConvolver(delta, 4096)
    x = np.random.default_rng(1).uniform(-1, 1, conv.hop_size).astype(np.float32)
    y = conv.apply(x)
    assert len(y) == len(x) + 63
    assert rel(y[: len(x)], x) < 1e-6
    assert np.max(np.abs(y[len(x):])) < 1e-6


def test_fused_matches_convolver_and_fp64(M):
    # FusedConvolverTests.swift:24-36 (128 taps, 8192-sample signal)
    rng = np.random.default_rng(2)
    h = rng.uniform(-1, 1, 128).astype(np.float32)
    x = rng.uniform(-1, 1, 8192).astype(np.float32)
    a = M.FusedConvolver(h, 4096).apply(x)
    b = M.Convolver(h, 4096).apply(x)
    assert np.array_equal(a, b)
    assert rel(a, O.conv64(x, h, 4096)) < 1e-6
    assert rel(a, O.ref_conv(x, h, 4096)) < 1e-5  # the reference algorithm in FP32


@pytest.mark.parametrize("K,fft,nx", [(1, 64, 1000), (31, 64, 200), (63, 64, 500), (33, 64, 1),
                                      (100, 256, 0), (255, 512, 5000), (1000, 2048, 70000),
                                      (4095, 8192, 100000), (129, 16384, 40000), (3000, 4096, 9999)])
def test_convolver_vs_fp64(M, K, fft, nx):
    rng = np.random.default_rng(K * 7 + nx)
    h = rng.standard_normal(K).astype(np.float32)
    x = rng.standard_normal(nx).astype(np.float32)
    y = M.Convolver(h, fft).apply(x)
    assert y.shape == (nx + K - 1,)
    ref = O.conv64(x, h, fft)
    if nx == 0:
        assert np.all(y == 0)
    else:
        assert rel(y, ref) < 2e-6, rel(y, ref)


def test_convolver_device_tensors(M):
    import torch
    rng = np.random.default_rng(3)
    h = rng.standard_normal(4095).astype(np.float32)
    x = rng.standard_normal(300000).astype(np.float32)
    conv = M.Convolver(h, 8192)
    yd = conv.apply(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert rel(yd.cpu().numpy(), O.conv64(x, h, 8192)) < 2e-6
    assert conv.block_size == 8192 and conv.hop_size == 8192 - 4095 + 1


def test_recommended_fft_size(M):
    assert M.Convolver.recommended_fft_size(100) == 128
    assert M.Convolver.recommended_fft_size(16384) is None


def test_convolver_preconditions(M):
    with pytest.raises(M.FFTError) as e:
        M.Convolver(np.ones(64, np.float32), 64)
    assert e.value.case == "invalidArgument"
    with pytest.raises(M.FFTError):
        M.FusedConvolver(np.ones(8, np.float32), 2048)


@pytest.mark.parametrize("K,fft,nx", [(9, 64, 60), (31, 64, 333), (255, 512, 4000), (4095, 8192, 70000)])
def test_adjoint_vs_fp64_analytic(M, K, fft, nx):
    rng = np.random.default_rng(K + nx)
    h = (rng.standard_normal(K) * np.exp(-np.arange(K) / 800.0)).astype(np.float32)
    x = rng.standard_normal(nx).astype(np.float32)
    t = rng.standard_normal(nx + K - 1).astype(np.float32)
    conv = M.Convolver(h, fft)
    g = (conv.apply(x).astype(np.float64) - t).astype(np.float32)
    dx, dh = conv.backward(x, g)
    rdx, rdh = O.conv_adjoint64(x, h, g)
    assert rel(dx, rdx) < 1e-5, rel(dx, rdx)
    assert rel(dh, rdh) < 1e-5, rel(dh, rdh)


def test_adjoint_vs_fp64_central_differences(M):
    """L = 0.5 ||x * h - t||^2: GPU gradients vs FP64 central differences of
    the FP64 oracle loss, within 1e-5 (relative L2 over the gradient)."""
    rng = np.random.default_rng(11)
    K, fft, nx = 9, 64, 80
    h = rng.standard_normal(K)
    x = rng.standard_normal(nx)
    t = rng.standard_normal(nx + K - 1)
    conv = M.Convolver(h.astype(np.float32), fft)
    y = conv.apply(x.astype(np.float32)).astype(np.float64)
    dx, dh = conv.backward(x.astype(np.float32), (y - t).astype(np.float32))

    def loss(x_, h_):
        return 0.5 * np.sum((O.conv64(x_, h_, fft) - t) ** 2)

    eps = 1e-5
    fdx = np.array([(loss(x + eps * e, h) - loss(x - eps * e, h)) / (2 * eps) for e in np.eye(nx)])
    fdh = np.array([(loss(x, h + eps * e) - loss(x, h - eps * e)) / (2 * eps) for e in np.eye(K)])
    assert rel(dx, fdx) < 1e-5, rel(dx, fdx)
    assert rel(dh, fdh) < 1e-5, rel(dh, fdh)


def test_config4_full_size_adjoint_identities(M):
    """2^24-sample signal, 4095 taps, fft 8192 on the device: y against the
    FP64 OLA oracle; dx and dh through the adjoint identities
    <conv(x), g> = <x, dx> and <conv_h(x), g> = <h, dh> (size-independent)."""
    import torch
    from metalfft_b200 import workloads
    x, h, t = workloads.conv_workload(nx=1 << 24)
    conv = M.Convolver(h, 8192)
    xd = torch.from_numpy(x).cuda()
    y = conv.apply(xd)
    g = y - torch.from_numpy(t).cuda()
    dx, dh = conv.backward(xd, g)
    torch.cuda.synchronize()
    yh = y.cpu().numpy()
    assert rel(yh, O.conv64(x, h, 8192)) < 2e-6
    gh = g.cpu().numpy().astype(np.float64)
    lhs = float(np.dot(yh.astype(np.float64), gh))
    assert abs(lhs - float(np.dot(x.astype(np.float64), dx.cpu().numpy().astype(np.float64)))) < 1e-5 * abs(lhs) + 1e-3
    assert abs(lhs - float(np.dot(h.astype(np.float64), dh.cpu().numpy().astype(np.float64)))) < 1e-5 * abs(lhs) + 1e-3


# ---- Correlator ------------------------------------------------------------

@pytest.mark.parametrize("fft,na,nb", [(256, 200, 300), (1024, 1024, 10), (4096, 5000, 4000), (64, 0, 10)])
def test_correlator_cross(M, fft, na, nb):
    rng = np.random.default_rng(fft + na)
    a = rng.standard_normal(na).astype(np.float32)
    b = rng.standard_normal(nb).astype(np.float32)
    r = M.Correlator(fft).cross(a, b)
    ref = O.corr64(a, b, fft)
    assert np.max(np.abs(r - ref)) <= 2e-6 * max(1.0, np.max(np.abs(ref))) * np.sqrt(fft)


def test_autocorrelation_peak_is_energy(M):
    x = np.random.default_rng(5).standard_normal(100).astype(np.float32)
    r = M.Correlator(256).auto(x)
    assert abs(r[0] - np.sum(x.astype(np.float64) ** 2)) < 1e-4 * np.sum(x ** 2)
    assert int(np.argmax(r)) == 0


# ---- golden fixtures (tests/golden/make_golden.py: the reference's host loops
# ---- transliterated to numpy over FP64 pocketfft, independent of oracle/)

def _golden(name):
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", name))


def test_golden_convolver_cases(M):
    """Convolver.apply and its adjoint on the reference's edge cases: an empty
    signal, shorter than one hop, K = 1, ending on a hop boundary, hop 2."""
    z = _golden("conv_golden.npz")
    for name in z["cases"]:
        x, h, y, t = z[name + "_x"], z[name + "_h"], z[name + "_y"], z[name + "_t"]
        conv = M.Convolver(h, int(z[name + "_fft"]))
        yg = conv.apply(x)
        assert yg.shape == y.shape, name
        if len(x) == 0:
            assert not yg.any()
            continue
        assert rel(yg, y) < 2e-6, (name, rel(yg, y))
        g = (y - t).astype(np.float32)
        dx, dh = conv.backward(x, g)
        rdx, rdh = O.conv_adjoint64(x, h, g)  # at the FP32 gradient the GPU saw
        assert rel(dx, rdx) < 1e-5 and rel(dh, rdh) < 1e-5, name
        assert rel(dx, z[name + "_dx"]) < 1e-5 and rel(dh, z[name + "_dh"]) < 1e-5, name


def test_golden_correlator_cases(M):
    z = _golden("corr_golden.npz")
    for name in z["cases"]:
        a, b, r = z[name + "_a"], z[name + "_b"], z[name + "_r"]
        out = M.Correlator(int(z[name + "_fft"])).cross(a, b)
        assert out.shape == r.shape, name
        scale = max(np.max(np.abs(r)), float(np.sum(a.astype(np.float64) ** 2)))
        assert np.max(np.abs(out - r)) <= 2e-6 * scale, name


def test_golden_analyzer_windows(M):
    z = _golden("analyzer_golden.npz")
    n = len(z["w_rect"])
    s = z["samples"]
    for key, wt in [("flattop", M.WindowType(M.WindowType.FLAT_TOP)), ("kaiser6", M.WindowType.kaiser(6.0)),
                    ("kaiser9", M.WindowType.kaiser(9.5)), ("rect", M.WindowType(M.WindowType.RECTANGULAR))]:
        an = M.FFTAnalyzer(n, 48000.0, wt)
        assert O.rel_rms(an.analyze(s[:n]).complex[None], z["X0_" + key][None]) < 2e-6, key
        assert O.rel_rms(an.analyze(s, offset=n + 17).complex[None], z["X1_" + key][None]) < 2e-6, key


# ---- FFTAnalyzer -----------------------------------------------------------

@pytest.mark.parametrize("kind", [0, 1, 2, 3, 5])
def test_analyzer_vs_fp64(M, kind):
    n = 2048
    s = np.random.default_rng(kind).standard_normal(3 * n).astype(np.float32)
    an = M.FFTAnalyzer(n, 48000.0, M.WindowType(kind))
    res = an.analyze(s, offset=n)
    w = O.window(kind, n)
    ref = np.fft.fft(s[n:2 * n].astype(np.float64) * w)
    assert O.rel_rms(res.complex[None], ref[None]) < 2e-6
    res0 = an.analyze(s[:n])
    assert O.rel_rms(res0.complex[None], np.fft.fft(s[:n].astype(np.float64) * w)[None]) < 2e-6
    with pytest.raises(M.FFTError):
        an.analyze(s, offset=2 * n + 1)


def test_analyzer_sine_peak_and_rms(M):
    n, fs = 1024, 1024.0
    k = np.arange(n)
    x = np.sin(2 * np.pi * 100 * k / n).astype(np.float32)
    res = M.FFTAnalyzer(n, fs, M.WindowType(M.WindowType.RECTANGULAR)).analyze(x)
    assert int(np.argmax(res.magnitudes[: n // 2])) == 100
    assert abs(res.bin_frequency(100) - 100.0) < 1e-9
    # Parseval: sqrt(sum |X|^2) / N = rms * sqrt(N) / sqrt(N)... = sqrt(sum x^2 / N)
    assert abs(res.rms - np.sqrt(np.sum(x.astype(np.float64) ** 2)) / np.sqrt(n)) < 1e-5


# ---- mixed sizes in one persistent launch ------------------------------------

def _check_mixed(M, classes, seed, inverse=False, sample=None):
    import torch
    mb = M.MixedBatch(classes)
    x = O.normal_c64((mb.points,), seed)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    mb.exec(xd, yd, M.INVERSE if inverse else M.FORWARD)
    torch.cuda.synchronize()
    assert M.lib.mfft_context_check(M.shared_context()) == 0
    y = yd.cpu().numpy()
    for n, c, off in mb.layout:
        idx = range(c) if sample is None else sorted(set([0, c - 1] + list(range(0, c, max(1, c // sample)))))
        for j in idx:
            seg = slice(off + j * n, off + (j + 1) * n)
            e = O.rel_rms(y[seg][None], O.truth(x[seg][None], inverse=inverse))
            assert e < (2e-6 if n <= 16384 else 3e-6), (n, j, e)


def test_mixed_small_set(M):
    classes = [(64, 3), (128, 1), (256, 17), (512, 2), (1024, 5), (2048, 1), (4096, 3), (8192, 2),
               (16384, 2), (1 << 15, 1), (1 << 16, 2), (1 << 17, 1), (1 << 18, 1), (1 << 19, 1), (1 << 20, 2)]
    _check_mixed(M, classes, seed=31)
    _check_mixed(M, classes, seed=32, inverse=True)


def test_mixed_more_tma_classes_than_groups(M):
    # ten 2^16 classes: the first eight move their tiles by TMA inside the
    # queue launch, the last two take the 16-byte-copy items of the same kernel
    classes = [(1 << 16, 1)] * 10 + [(64, 5), (1 << 15, 1)]
    _check_mixed(M, classes, seed=34)
    _check_mixed(M, classes, seed=35, inverse=True)


def test_mixed_config2_full(M):
    from metalfft_b200 import workloads
    classes = workloads.mixed_size_classes()
    assert sum(n * c for n, c in classes) <= 1 << 26
    _check_mixed(M, classes, seed=33, sample=3)


def test_mixed_host_arrays(M):
    classes = [(64, 5), (4096, 2), (1 << 16, 1)]
    mb = M.MixedBatch(classes)
    x = O.uniform_c64((mb.points,), 40)
    y = mb.forward(x)
    for n, c, off in mb.layout:
        for j in range(c):
            seg = slice(off + j * n, off + (j + 1) * n)
            assert O.rel_rms(y[seg][None], O.truth(x[seg][None])) < 3e-6


def test_mixed_in_place_matches_out_of_place(M):
    # in == out: a transform's row items, which write its output, start after
    # all of its column items have read its input (TMA classes alike)
    import torch
    classes = [(256, 7), (4096, 3), (8192, 2), (1 << 15, 1), (1 << 16, 2), (1 << 18, 1), (1 << 20, 2)]
    mb = M.MixedBatch(classes)
    x = torch.from_numpy(O.normal_c64((mb.points,), 41)).cuda()
    y = torch.empty_like(x)
    mb.exec(x, y, M.FORWARD)
    z = x.clone()
    mb.exec(z, z, M.FORWARD)
    torch.cuda.synchronize()
    assert torch.equal(y, z)


def test_mixed_graph_replay_matches_exec(M):
    # config 2 runs as one CUDA graph per step: the captured counter reset and
    # queue launch (tensor maps passed by value) replay to the same bits as a
    # direct call, twice in a row
    import torch
    classes = [(64, 9), (2048, 3), (16384, 2), (1 << 16, 1), (1 << 20, 2)]
    mb = M.MixedBatch(classes)
    x = torch.from_numpy(O.normal_c64((mb.points,), 43)).cuda()
    y = torch.empty_like(x)
    mb.exec(x, y)
    ref = y.clone()
    y.zero_()
    g = mb.capture(x, y)
    for _ in range(2):
        y.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(y, ref)
    del g
