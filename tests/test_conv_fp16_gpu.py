"""FusedConvolver's FP16 precision modes (DSP/FusedConvolver.swift:27-36,
Resources/fft_fused_convolve_fp16.metal) on the GPU: the reference's own
thresholds against the FP32 mode (FusedConvolverTests.swift:38-64) and the
same bounds against the FP64 oracle."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# FusedConvolverTests.swift:40-50
BOUND = {"float16Pure": 2e-2, "float16Storage": 1e-3, "float16Mixed": 2e-2}
MODES = list(BOUND)


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("mode", MODES)
def test_fp16_mode_matches_fp32(M, mode):
    # FusedConvolverTests.swift:52-64: 64 taps, fftSize + 500 samples, U[-1, 1)
    rng = np.random.default_rng(11)
    h = rng.uniform(-1, 1, 64).astype(np.float32)
    x = rng.uniform(-1, 1, 4096 + 500).astype(np.float32)
    ref = M.FusedConvolver(h, 4096, precision="float32").apply(x)
    out = M.FusedConvolver(h, 4096, precision=mode).apply(x)
    assert out.shape == ref.shape == (len(x) + 63,)
    assert rel(out, ref) < BOUND[mode], (mode, rel(out, ref))
    assert rel(out, O.conv64(x, h, 4096)) < BOUND[mode]


@pytest.mark.parametrize("mode", MODES)
def test_fp16_delta_filter_is_identity(M, mode):
    # FusedConvolverTests.swift:11-22 in each mode
    delta = np.zeros(64, np.float32)
    delta[0] = 1
    conv = M.FusedConvolver(delta, 4096, precision=mode)
    x = np.random.default_rng(12).uniform(-1, 1, conv.hop_size).astype(np.float32)
    y = conv.apply(x)
    assert y.shape == (len(x) + 63,)
    assert rel(y[: len(x)], x) < BOUND[mode]
    assert np.max(np.abs(y[len(x):])) < 10 * BOUND[mode]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("K,nx,amp", [(128, 1 << 20, 1.0), (4000, 300000, 1.0), (1, 50000, 1.0), (512, 200000, 4.0),
                                      (2000, 7, 1.0)])
def test_fp16_long_signals_vs_fp64(M, mode, K, nx, amp):
    # many walkers, warm-up blocks at every range start (K = 4000: hop 97),
    # a one-tap kernel, a 4x louder signal, a signal shorter than one hop
    rng = np.random.default_rng(K + nx)
    h = (rng.uniform(-1, 1, K) / np.sqrt(K / 64.0)).astype(np.float32)
    x = (amp * rng.uniform(-1, 1, nx)).astype(np.float32)
    y = M.FusedConvolver(h, 4096, precision=mode).apply(x)
    assert y.shape == (nx + K - 1,)
    assert np.all(np.isfinite(y))
    assert rel(y, O.conv64(x, h, 4096)) < BOUND[mode], (mode, rel(y, O.conv64(x, h, 4096)))


@pytest.mark.parametrize("mode", MODES)
def test_fp16_device_matches_host_and_backward_stays_fp32(M, mode):
    import torch
    rng = np.random.default_rng(13)
    h = rng.uniform(-1, 1, 300).astype(np.float32)
    x = rng.uniform(-1, 1, 123457).astype(np.float32)
    conv = M.FusedConvolver(h, 4096, precision=mode)
    yh = conv.apply(x)
    yd = conv.apply(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(yh, yd.cpu().numpy())
    assert np.array_equal(yh, conv.apply(x))  # deterministic
    g = rng.standard_normal(len(yh)).astype(np.float32)
    dx, dh = conv.backward(x, g)
    dx32, dh32 = M.FusedConvolver(h, 4096).backward(x, g)
    assert np.array_equal(dx, dx32) and np.array_equal(dh, dh32)


def test_fp16_precision_errors(M):
    h = np.ones(8, np.float32)
    with pytest.raises(M.FFTError) as e:
        M.FusedConvolver(h, 4096, precision="float16")
    assert e.value.case == "invalidArgument"
    c = M.Convolver(h, 2048)
    with pytest.raises(M.FFTError) as e:
        M._check(M.lib.mfft_conv_set_precision(c._h, 2))  # FP16 modes are fftSize 4096 only
    assert e.value.case == "invalidArgument" and e.value.got == 2048
    c4 = M.Convolver(h, 4096)
    for bad in (-1, 4):
        with pytest.raises(M.FFTError):
            M._check(M.lib.mfft_conv_set_precision(c4._h, bad))
    with pytest.raises(M.FFTError):
        M._check(M.lib.mfft_conv_set_precision(ctypes.c_void_p(), 1))
    # back to FP32 on the same handle: bit-identical to a fresh FP32 convolver
    x = np.random.default_rng(14).uniform(-1, 1, 10000).astype(np.float32)
    M._check(M.lib.mfft_conv_set_precision(c4._h, 2))
    M._check(M.lib.mfft_conv_set_precision(c4._h, 0))
    assert np.array_equal(c4.apply(x), M.Convolver(h, 4096).apply(x))
