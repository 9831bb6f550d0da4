"""Adjoint (backward) of the batched FFT through the C ABI
(mfft_exec_c2c_backward), checked three ways against FP64:

  - as a transform: the adjoint of the unscaled forward is n * inverse, the
    adjoint of the 1/n inverse is forward / n (the reference's conventions,
    Sources/MetalFFT/FFT/MetalFFT.swift:56-65, fft_multisize.metal:70);
  - the inner-product identity Re<F x, g> = Re<x, F^H g>;
  - FP64 central differences of L(x) = 0.5 ||T(x) - t||^2 for T = forward and
    T = inverse, at sampled input components (real and imaginary parts),
    within 1e-5 of the largest gradient component.
The reference has no backward pass, so these bars are FP64 ones."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [64, 256, 1024, 4096, 8192, 16384, 1 << 15, 1 << 17, 1 << 20]


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


def tol(n):
    return 2e-6 if n <= 16384 else 3e-6


@pytest.mark.parametrize("n", SIZES)
def test_backward_is_the_conjugate_transpose(M, n):
    b = 3 if n <= 16384 else 2
    g = O.normal_c64((b, n), seed=8000 + n)
    f = M.MetalFFT(n)
    g64 = g.astype(np.complex128)
    # adjoint of the forward: n * inverse = unscaled conjugate transform
    gx = f.backward_batch(g, M.FORWARD)
    assert O.rel_rms(gx, n * np.fft.ifft(g64, axis=-1)) < tol(n)
    # adjoint of the inverse: forward / n
    gx = f.backward_batch(g, M.INVERSE)
    assert O.rel_rms(gx, np.fft.fft(g64, axis=-1) / n) < tol(n)


@pytest.mark.parametrize("n", [256, 4096, 1 << 16])
def test_inner_product_identity(M, n):
    x = O.normal_c64((2, n), seed=8100 + n)
    g = O.normal_c64((2, n), seed=8200 + n)
    f = M.MetalFFT(n)
    for d in (M.FORWARD, M.INVERSE):
        y = (f.forward_batch(x) if d == M.FORWARD else f.inverse_batch(x)).astype(np.complex128)
        ag = f.backward_batch(g, d).astype(np.complex128)
        lhs = np.vdot(g.astype(np.complex128), y).real      # Re <T x, g>
        rhs = np.vdot(ag, x.astype(np.complex128)).real     # Re <x, T^H g>
        scale = np.linalg.norm(y) * np.linalg.norm(g)
        assert abs(lhs - rhs) <= 2e-6 * scale, (d, lhs, rhs)


@pytest.mark.parametrize("n", [256, 4096, 1 << 17])
@pytest.mark.parametrize("direction", ["forward", "inverse"])
def test_central_differences(M, n, direction):
    rng = np.random.default_rng(8300 + n)
    x = O.uniform_c64((n,), seed=8400 + n)
    t = O.uniform_c64((n,), seed=8500 + n).astype(np.complex128)
    f = M.MetalFFT(n)
    fwd = direction == "forward"
    d = M.FORWARD if fwd else M.INVERSE

    def T64(v):
        return np.fft.fft(v) if fwd else np.fft.ifft(v)

    def loss(v):
        r = T64(v) - t
        return 0.5 * float(np.vdot(r, r).real)

    # GPU: y = T(x), g = dL/dy = y - t, dL/dx = backward(g)
    y = f.forward(x) if fwd else f.inverse(x)
    g = (y.astype(np.complex128) - t).astype(np.complex64)
    grad = f.backward(g, d).astype(np.complex128)
    x64 = x.astype(np.complex128)
    # L is quadratic in x, so a central difference has no truncation error at
    # any step: a large step keeps the FP64 rounding (~eps L / h) negligible
    h = 0.5
    idx = rng.choice(n, 12, replace=False)
    fd = []
    for j in idx:
        comp = []
        for unit in (1.0, 1j):
            e = np.zeros(n, np.complex128)
            e[j] = unit * h
            comp.append((loss(x64 + e) - loss(x64 - e)) / (2 * h))
        fd.append(comp[0] + 1j * comp[1])
    fd = np.array(fd)
    # analytic FP64 adjoint at the same point
    r = T64(x64) - t
    exact = (n * np.fft.ifft(r)) if fwd else (np.fft.fft(r) / n)
    big = np.max(np.abs(exact))
    assert np.max(np.abs(fd - exact[idx])) <= 1e-8 * big  # the FD estimate itself
    assert np.max(np.abs(grad[idx] - fd)) <= 1e-5 * big, np.max(np.abs(grad[idx] - fd)) / big
    assert O.rel_rms(grad, exact) < 1e-5


def test_backward_device_tensors_and_in_place(M):
    import torch
    n, b = 4096, 5
    g = torch.from_numpy(O.normal_c64((b, n), seed=8600)).cuda()
    f = M.MetalFFT(n)
    out = torch.empty_like(g)
    f.exec_backward(g, out, b, M.FORWARD)
    ref = n * np.fft.ifft(g.cpu().numpy().astype(np.complex128), axis=-1)
    assert O.rel_rms(out.cpu().numpy(), ref) < 2e-6
    # in place gives the same bits
    h = g.clone()
    f.exec_backward(h, h, b, M.FORWARD)
    torch.cuda.synchronize()
    assert torch.equal(h, out)
    # the adjoint of the forward is exactly n x the inverse (power-of-two scales)
    inv = torch.empty_like(g)
    f.exec(g, inv, b, M.INVERSE)
    assert torch.equal(out, inv * n)
