"""Four-step FFT (n = 2^15 .. 2^20) on every admissible split n = n1 x n2
(64 <= n1 <= 1024, 128 <= n2 <= 1024), and the split autotuner.  The
reference fixes one split per size (MetalContext.swift:57-66); every split
here must give the same transform: FP32 within 3e-6 rel RMS of the FP64
oracle, forward, inverse and the adjoint (backward) entry."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

BIG = [1 << 15, 1 << 16, 1 << 17, 1 << 18, 1 << 19, 1 << 20]
TOL_BIG = 3e-6


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


@pytest.fixture
def ctx(M):
    """A private context, so that installed splits do not leak into other tests."""
    h = ctypes.c_void_p()
    assert M.lib.mfft_context_create(0, ctypes.byref(h)) == 0
    yield h
    M.lib.mfft_context_destroy(h)


def cases():
    out = []
    for n in BIG:
        logn = n.bit_length() - 1
        for l1 in range(6, 11):
            if 7 <= logn - l1 <= 10:
                out.append((n, 1 << l1))
    return out


@pytest.mark.parametrize("n,n1", cases())
def test_every_split_matches_fp64(M, n, n1):
    b = 3 if n <= (1 << 18) else 2
    x = O.normal_c64((b, n), seed=n + n1)
    f = M.MetalFFT(n)
    f.set_split(n1)
    assert f.split == (n1, n // n1)
    assert O.rel_rms(f.forward_batch(x), O.truth(x)) < TOL_BIG
    assert O.rel_rms(f.inverse_batch(x), O.truth(x, inverse=True)) < TOL_BIG


@pytest.mark.parametrize("n,n1", [(1 << 16, 128), (1 << 18, 1024), (1 << 17, 256), (1 << 19, 512)])
def test_split_device_batch_and_adjoint(M, n, n1):
    """Odd device batch (the TMA tiles' last boxes) in place, and the backward
    entry: the adjoint of the forward transform is n times the inverse."""
    import torch
    b = 5
    x = O.normal_c64((b, n), seed=7 * n + n1)
    f = M.MetalFFT(n)
    f.set_split(n1)
    xd = torch.from_numpy(x).cuda()
    z = xd.clone()
    f.exec(z, z, b, M.FORWARD)
    torch.cuda.synchronize()
    assert O.rel_rms(z.cpu().numpy(), O.truth(x)) < TOL_BIG
    g = f.backward_batch(x, M.FORWARD)
    assert O.rel_rms(g, O.truth(x, inverse=True) * n) < TOL_BIG
    gi = f.backward_batch(x, M.INVERSE)  # adjoint of the inverse = forward / n
    assert O.rel_rms(gi, O.truth(x) / n) < TOL_BIG


def test_splits_listed_and_invalid_split_rejected(M):
    assert M.MetalFFT.splits(1 << 15) == [64, 128, 256]
    assert M.MetalFFT.splits(1 << 20) == [1024]
    assert M.MetalFFT.splits(4096) == []
    f = M.MetalFFT(1 << 16)
    before = f.split
    with pytest.raises(M.FFTError):
        f.set_split(32)   # n2 = 2048 > 1024
    with pytest.raises(M.FFTError):
        f.set_split(100)  # not a power of two
    assert f.split == before
    g = M.MetalFFT(4096)
    assert g.split == (0, 0)
    with pytest.raises(M.FFTError):
        g.set_split(64)


@pytest.mark.parametrize("n", [1 << 17, 1 << 18])
def test_autotune_installs_split_in_context(M, ctx, n):
    f = M.MetalFFT(n, context=ctx)
    n1 = f.autotune_split(batch=64)
    assert n1 in M.MetalFFT.splits(n)
    assert f.split == (n1, n // n1)
    g = M.MetalFFT(n, context=ctx)  # later plans of the size in the context take it
    assert g.split == (n1, n // n1)
    x = O.normal_c64((2, n), seed=n + 5)
    assert O.rel_rms(g.forward_batch(x), O.truth(x)) < TOL_BIG


def test_split_cache_file_and_mixed_batch(M, ctx, tmp_path, monkeypatch):
    """A context reads its four-step splits from $MFFT_TUNE_CACHE ("n n1 0 0"
    lines); plans and a mixed launch built in it run those splits, here the
    item kernel's 16-byte-copy path (n2 = 128 or n1 = 128 below 256) and a
    TMA split other than the default, and match FP64."""
    import torch
    cache = tmp_path / "tune.txt"
    cache.write_text("131072 128 0 0\n65536 512 0 0\n262144 1024 0 0\n")
    monkeypatch.setenv("MFFT_TUNE_CACHE", str(cache))
    assert M.MetalFFT(1 << 17, context=ctx).split == (128, 1024)
    assert M.MetalFFT(1 << 16, context=ctx).split == (512, 128)
    assert M.MetalFFT(1 << 18, context=ctx).split == (1024, 256)
    sizes = [(4096, 3), (1 << 17, 2), (1 << 16, 3), (1 << 18, 1), (1 << 15, 2)]
    mb = M.MixedBatch(sizes, context=ctx)
    x = O.normal_c64((mb.points,), seed=11)
    xd = torch.from_numpy(x).cuda()
    for d in (M.FORWARD, M.INVERSE):
        y = torch.empty_like(xd)
        mb.exec(xd, y, d)
        torch.cuda.synchronize()
        Y = y.cpu().numpy()
        for (m, c, off) in mb.layout:
            seg = x[off:off + m * c].reshape(c, m)
            got = Y[off:off + m * c].reshape(c, m)
            assert O.rel_rms(got, O.truth(seg, inverse=d == M.INVERSE)) < TOL_BIG, (m, d)
