"""Parity of the tcgen05 DFT-as-matmul FFT (N = 4096) with the FP64 oracle:
the B200 form of the reference's fft_4096_ct_mma (src/fft_4096_ct_mma.metal
:88-206), checked like DemoComparisonTests.swift:23-112 (impulse -> ones, all
variants agree) but against FP64 with the split-FP16 bar of <= 3e-6 rel RMS."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 4096
TOL_SPLIT = 3e-6
TOL_BF16 = 2e-2


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


@pytest.mark.parametrize("batch", [1, 7, 300, 1000])
def test_split_fp16_forward_inverse(M, batch):
    x = O.normal_c64((batch, N), seed=500 + batch)
    f = M.MetalFFT(N)
    y = f.forward_batch(x, tc_variant=M.TC_FP16_SPLIT3)
    assert O.rel_rms(y, O.truth(x)) < TOL_SPLIT
    yi = f.inverse_batch(x, tc_variant=M.TC_FP16_SPLIT3)
    assert O.rel_rms(yi, O.truth(x, inverse=True)) < TOL_SPLIT


@pytest.mark.parametrize("tc", ["split", "bf16"])
def test_many_lines_per_cta(M, tc):
    """3000 lines: about 20 per persistent CTA, so every ring of the
    warp-specialised kernel (operand buffers, accumulator slots, line scales)
    wraps several times; every line against FP64."""
    x = O.normal_c64((3000, N), seed=612)
    x[1234] *= np.float32(1e12)  # one line far from the others: its own scale
    variant = M.TC_FP16_SPLIT3 if tc == "split" else M.TC_BF16
    bar = TOL_SPLIT if tc == "split" else TOL_BF16
    f = M.MetalFFT(N)
    y = f.forward_batch(x, tc_variant=variant)
    ref = O.truth(x)
    err = np.array([O.rel_rms(y[i:i + 1], ref[i:i + 1]) for i in range(0, 3000, 1)])
    assert err.max() < bar, (int(err.argmax()), err.max())
    yi = f.inverse_batch(x, tc_variant=variant)
    assert O.rel_rms(yi[::7], O.truth(x[::7], inverse=True)) < bar


def test_bf16_variant(M):
    x = O.normal_c64((64, N), seed=77)
    y = M.MetalFFT(N).forward_batch(x, tc_variant=M.TC_BF16)
    e = O.rel_rms(y, O.truth(x))
    assert e < TOL_BF16, e


def test_impulse_and_extreme_magnitudes(M):
    # DemoComparisonTests.swift:89-112: impulse -> all ones; plus lines whose
    # scale is far from 1 (per-line power-of-two scaling) and an all-zero line
    f = M.MetalFFT(N)
    x = np.zeros((5, N), np.complex64)
    x[0, 0] = 1
    x[1] = O.normal_c64((1, N), seed=1)[0] * np.float32(1e-30)
    x[2] = O.normal_c64((1, N), seed=2)[0] * np.float32(1e30)
    x[4] = O.uniform_c64((1, N), seed=3)[0]
    y = f.forward_batch(x, tc_variant=M.TC_FP16_SPLIT3)
    assert np.max(np.abs(y[0] - 1)) < 1e-6
    ref = O.truth(x)
    for i in [1, 2, 4]:
        assert O.rel_rms(y[i:i + 1], ref[i:i + 1]) < TOL_SPLIT, i
    assert np.all(y[3] == 0)


def test_variants_agree_with_fp32_stockham(M):
    # DemoComparisonTests.swift:64-86 (all FFT variants agree)
    x = O.uniform_c64((33, N), seed=9)
    f = M.MetalFFT(N)
    a = f.forward_batch(x)
    b = f.forward_batch(x, tc_variant=M.TC_FP16_SPLIT3)
    assert O.rel_rms(b, a.astype(np.complex128)) < 2 * TOL_SPLIT


def test_device_tensors_in_place(M):
    import torch
    x = O.normal_c64((200, N), seed=10)
    t = torch.from_numpy(x).cuda()
    f = M.MetalFFT(N)
    f.exec(t, t, 200, M.FORWARD, M.TC_FP16_SPLIT3)
    torch.cuda.synchronize()
    assert O.rel_rms(t.cpu().numpy(), O.truth(x)) < TOL_SPLIT
    assert M.lib.mfft_context_check(M.shared_context()) == 0


def test_tc_rejects_other_sizes(M):
    with pytest.raises(M.FFTError) as e:
        M.MetalFFT(1024).forward_batch(np.zeros((1, 1024), np.complex64), tc_variant=M.TC_FP16_SPLIT3)
    assert e.value.case == "unsupportedFFTSize"
