"""Parity of the CUDA batched FFT (through libmfft's C ABI) with the FP64
oracle, following the reference's own tests (Tests/MetalFFTTests/
MetalFFTTests.swift) with tighter bars: FP32 <= 2e-6 rel RMS for N <= 16384
against FP64 (the reference: 1e-4 against vDSP), 3e-6 for the four-step sizes."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384]
BIG = [1 << 15, 1 << 16, 1 << 17, 1 << 18, 1 << 19, 1 << 20]
TOL = 2e-6       # FP32, N <= 16384, rel RMS vs FP64
TOL_BIG = 3e-6   # four-step sizes


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


def tol(n):
    return TOL if n <= 16384 else TOL_BIG


@pytest.mark.parametrize("n", SIZES)
def test_all_sizes_impulse(M, n):
    # MetalFFTTests.swift:11-23
    x = np.zeros(n, np.complex64)
    x[0] = 1
    y = M.MetalFFT(n).forward(x)
    assert np.max(np.abs(y.real - 1)) < 1e-6 and np.max(np.abs(y.imag)) < 1e-6


@pytest.mark.parametrize("n", SIZES + BIG)
def test_random_vs_fp64(M, n):
    # MetalFFTTests.swift:25-35, against FP64 instead of vDSP
    b = 3 if n <= 16384 else 2
    x = O.uniform_c64((b, n), seed=1000 + n)
    f = M.MetalFFT(n)
    y = f.forward_batch(x)
    assert O.rel_rms(y, O.truth(x)) < tol(n)
    xi = f.inverse_batch(x)
    assert O.rel_rms(xi, O.truth(x, inverse=True)) < tol(n)


@pytest.mark.parametrize("n", SIZES)
def test_every_registered_variant(M, n):
    x = O.normal_c64((5, n), seed=2000 + n)
    ref = O.truth(x)
    f = M.MetalFFT(n)
    xs = O.normal_c64((1000, n), seed=2100 + n) if n <= 1024 else x  # several groups per CTA
    refs = O.truth(xs)
    for var in M.MetalFFT.variants(n):
        f.set_kernel(*var)
        assert O.rel_rms(f.forward_batch(x), ref) < TOL, var
        assert O.rel_rms(f.inverse_batch(x), O.truth(x, inverse=True)) < TOL, var
        assert O.rel_rms(f.forward_batch(xs), refs) < TOL, var


@pytest.mark.parametrize("n", [64, 4096, 16384, 1 << 20])
def test_round_trip(M, n):
    x = O.uniform_c64((2, n), seed=3000 + n)
    f = M.MetalFFT(n)
    z = f.inverse_batch(f.forward_batch(x))
    assert O.rel_rms(z, x.astype(np.complex128)) < 2 * tol(n)


def test_single_matches_batch_bitwise(M):
    # MetalFFTTests.swift:51-65 (the reference allows 1e-4; same kernel here)
    n = 512
    x = O.uniform_c64((2, n), seed=4)
    f = M.MetalFFT(n)
    yb = f.forward_batch([x[0], x[1]])
    assert np.array_equal(yb[0], f.forward(x[0]))
    assert np.array_equal(yb[1], f.forward(x[1]))


def test_cosine_peak_bin(M):
    # MetalFFTTests.swift:37-49
    n = 1024
    k = np.arange(n)
    x = np.cos(2 * np.pi * 100 * k / n).astype(np.complex64)
    y = M.MetalFFT(n).forward(x)
    assert int(np.argmax(np.abs(y[: n // 2]) ** 2)) == 100


def test_golden_fixtures(M):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "fft_golden.npz"))
    for n in [64, 512, 4096]:
        f = M.MetalFFT(n)
        assert O.rel_rms(f.forward_batch(z["x_%d" % n]), z["X_%d" % n]) < TOL
        assert O.rel_rms(f.inverse_batch(z["x_%d" % n]), z["Xi_%d" % n]) < TOL


def test_forward_into_and_multichannel(M):
    n = 256
    x = O.uniform_c64((4, n), seed=9)
    f = M.MetalFFT(n)
    out = np.zeros(3, np.complex64)
    f.forward_into(x[0], out)
    assert out.shape == (n,) and O.rel_rms(out[None], O.truth(x[:1])) < TOL
    mc = M.MultiChannelFFT(4, n)
    assert O.rel_rms(mc.forward(x), O.truth(x)) < TOL
    assert O.rel_rms(mc.inverse(x), O.truth(x, inverse=True)) < TOL
    with pytest.raises(M.FFTError):
        mc.forward(x[:3])


def test_device_tensors_and_in_place(M):
    import torch
    n = 4096
    x = O.normal_c64((64, n), seed=10)
    f = M.MetalFFT(n)
    t = torch.from_numpy(x).cuda()
    y = f.forward_batch(t)
    assert y.is_cuda
    assert O.rel_rms(y.cpu().numpy(), O.truth(x)) < TOL
    f.exec(t, t, 64)  # in place
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), y.cpu().numpy())


def test_errors_mirror_fft_error(M):
    with pytest.raises(M.FFTError) as e:
        M.MetalFFT(100)
    assert e.value.case == "unsupportedFFTSize" and e.value.expected == 100
    for bad in [32, 3 << 10, 1 << 21]:
        with pytest.raises(M.FFTError):
            M.MetalFFT(bad)
    f = M.MetalFFT(256)
    with pytest.raises(M.FFTError) as e:
        f.forward(np.zeros(255, np.complex64))
    assert e.value.case == "invalidInputSize" and (e.value.expected, e.value.got) == (256, 255)
    with pytest.raises(M.FFTError) as e:
        f.forward_batch([np.zeros(256, np.complex64), np.zeros(200, np.complex64)])
    assert e.value.case == "batchInputSize" and e.value.batch_index == 1
    assert f.forward_batch([]).shape == (0, 256)


def test_config1_batch256_forward_inverse(M):
    """N=4096, batch 256, U[-1,1): forward, inverse, round trip vs FP64."""
    n, b = 4096, 256
    x = O.uniform_c64((b, n), seed=12345)
    f = M.MetalFFT(n)
    X = f.forward_batch(x)
    assert O.rel_rms(X, O.truth(x)) < TOL
    xr = f.inverse_batch(X)
    assert O.rel_rms(xr, x.astype(np.complex128)) < TOL


def test_config3_full_batch_properties(M):
    """N=4096 x 16384 (512 MiB): sampled rows vs FP64, and linearity of the
    whole batch (a size-independent property)."""
    import torch
    n, b = 4096, 16384
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(b, n, dtype=torch.complex64, device="cuda", generator=g)
    yv = torch.randn(b, n, dtype=torch.complex64, device="cuda", generator=g)
    f = M.MetalFFT(n)
    X = f.forward_batch(x)
    Y = f.forward_batch(yv)
    rows = torch.randint(0, b, (32,), generator=torch.Generator().manual_seed(1))
    xs = x[rows].cpu().numpy()
    assert O.rel_rms(X[rows].cpu().numpy(), O.truth(xs)) < TOL
    Z = f.forward_batch(x + 2 * yv)
    lin = torch.linalg.vector_norm(Z - (X + 2 * Y)) / torch.linalg.vector_norm(Z)
    assert float(lin) < 4e-7 * 10
    # last rows (tail of the grid)
    assert O.rel_rms(X[-3:].cpu().numpy(), O.truth(x[-3:].cpu().numpy())) < TOL


def test_autotune_picks_a_registered_variant(M):
    import ctypes
    r, fpb, stg = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = M.lib.mfft_autotune(M.shared_context(), 1024, 4096, ctypes.byref(r), ctypes.byref(fpb),
                             ctypes.byref(stg))
    assert st == 0 and (r.value, fpb.value, stg.value) in M.MetalFFT.variants(1024)
    f = M.MetalFFT(1024)
    ki = f.kernel_info
    assert (ki["radix"], ki["lines_per_cta"], ki["stages"]) == (r.value, fpb.value, stg.value)
    x = O.normal_c64((3, 1024), seed=77)
    assert O.rel_rms(f.forward_batch(x), O.truth(x)) < TOL


def test_captured_graph_matches_direct_exec(M):
    """MetalFFT.capture: forward + inverse of N=4096 x 256 in one CUDA graph
    gives bit-identical results to the same two launches made directly, on
    every replay (the config-1 step)."""
    import torch
    n, b = 4096, 256
    x0 = torch.from_numpy(O.uniform_c64((b, n), seed=321)).cuda()
    f = M.MetalFFT(n)
    y_ref = torch.empty_like(x0)
    r_ref = torch.empty_like(x0)
    f.exec(x0, y_ref, b, M.FORWARD)
    f.exec(y_ref, r_ref, b, M.INVERSE)
    x = x0.clone()
    y = torch.empty_like(x)
    r = torch.empty_like(x)
    g = f.capture([(x, y, b, M.FORWARD), (y, r, b, M.INVERSE)])
    for _ in range(3):
        y.zero_()
        r.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(y, y_ref) and torch.equal(r, r_ref)
    assert O.rel_rms(y.cpu().numpy(), O.truth(x0.cpu().numpy())) < TOL


@pytest.mark.parametrize("n,b", [(1 << 15, 1030), (1 << 20, 35)])
def test_fourstep_batch_spans_scratch_chunks(M, n, b):
    """A four-step batch larger than the plan's intermediate (2^25 points)
    runs as several column/row pass pairs: lines on both sides of the chunk
    boundary must match FP64, forward and inverse, and in place."""
    import torch
    x = O.normal_c64((b, n), seed=n + b)
    f = M.MetalFFT(n)
    xd = torch.from_numpy(x).cuda()
    y = torch.empty_like(xd)
    f.exec(xd, y, b, M.FORWARD)
    torch.cuda.synchronize()
    assert M.lib.mfft_context_check(M.shared_context()) == 0
    chunk = (1 << 25) // n
    rows = sorted({0, 1, chunk - 1, chunk, min(chunk + 1, b - 1), b - 1})
    Y = y.cpu().numpy()
    ref = O.truth(x[rows])
    for i, j in enumerate(rows):
        assert O.rel_rms(Y[j][None], ref[i][None]) < TOL_BIG, j
    z = y.clone()
    f.exec(z, z, b, M.INVERSE)  # in place
    torch.cuda.synchronize()
    assert O.rel_rms(z.cpu().numpy(), x.astype(np.complex128)) < TOL_BIG


def test_misaligned_device_buffer_is_rejected(M):
    """Device buffers must be 16-byte aligned; an 8-byte-aligned view is an
    invalidArgument error raised before anything is launched."""
    import torch
    n = 1 << 16
    f = M.MetalFFT(n)
    base = torch.zeros(n + 1, dtype=torch.complex64, device="cuda")
    view = base[1:]
    assert view.data_ptr() % 16 == 8
    out = torch.empty(n, dtype=torch.complex64, device="cuda")
    with pytest.raises(M.FFTError) as e:
        f.exec(view, out, 1, M.FORWARD)
    assert e.value.case == "invalidArgument"


@pytest.mark.parametrize("n", SIZES)
def test_real_input_fft_matches_fp64(M, n):
    """forward_real: n/2 + 1 bins of the FFT of real lines (odd batch: the
    last line has no partner); inverse_real recovers the lines."""
    b = 7
    x = np.random.default_rng(n).standard_normal((b, n)).astype(np.float32)
    f = M.MetalFFT(n)
    X = f.forward_real(x)
    assert X.shape == (b, n // 2 + 1)
    ref = O.truth(x.astype(np.complex64))[:, : n // 2 + 1]
    assert O.rel_rms(X, ref) < TOL
    xr = f.inverse_real(X)
    assert xr.shape == (b, n)
    assert float(np.linalg.norm(xr - x) / np.linalg.norm(x)) < TOL


def test_real_input_fft_device_and_errors(M):
    import torch
    n = 4096
    x = torch.randn(9, n, device="cuda")
    f = M.MetalFFT(n)
    X = f.forward_real(x)
    assert X.is_cuda and X.shape == (9, n // 2 + 1)
    assert np.array_equal(X.cpu().numpy(), f.forward_real(x.cpu().numpy()))
    back = f.inverse_real(X)
    assert float(torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x)) < TOL
    with pytest.raises(M.FFTError) as e:
        M.MetalFFT(1 << 16).forward_real(np.zeros(1 << 16, np.float32))
    assert e.value.case == "unsupportedFFTSize"
    with pytest.raises(M.FFTError) as e:
        f.forward_real(np.zeros(n - 1, np.float32))
    assert e.value.case == "invalidInputSize"


@pytest.mark.parametrize("kind,n,b", [("c2c", 4096, 2000), ("c2c", 1 << 20, 5), ("c2c", 64, 70001),
                                      ("tc", 4096, 1500), ("r2c", 16384, 1001), ("c2r", 16384, 1001),
                                      ("r2c", 4096, 4097)])
def test_host_arrays_across_staging_chunks(M, kind, n, b):
    # host-array calls move through 16 MiB staging chunks on separate upload /
    # download streams; every chunk's result equals the device-pointer call
    import ctypes
    import torch
    f = M.MetalFFT(n)
    rng = np.random.default_rng(n + b)
    P = lambda a: ctypes.c_void_p(a.data_ptr())  # noqa: E731
    if kind in ("c2c", "tc"):
        x = torch.from_numpy(rng.standard_normal((b, n, 2), dtype=np.float32)).view(torch.complex64)[..., 0]
        shape_out, dt_out = (b, n), torch.complex64
    elif kind == "r2c":
        x = torch.from_numpy(rng.standard_normal((b, n), dtype=np.float32))
        shape_out, dt_out = (b, n // 2 + 1), torch.complex64
    else:
        x = torch.from_numpy(rng.standard_normal((b, n // 2 + 1, 2), dtype=np.float32)).view(torch.complex64)[..., 0]
        shape_out, dt_out = (b, n), torch.float32
    x = x.contiguous()

    def run(src, dst, flags):
        if kind == "c2c":
            return M.lib.mfft_exec_c2c(f._plan, P(src), P(dst), b, M.FORWARD, flags, None)
        if kind == "tc":
            return M.lib.mfft_exec_c2c_tc(f._plan, P(src), P(dst), b, M.FORWARD, 1, flags, None)
        fn = M.lib.mfft_exec_r2c if kind == "r2c" else M.lib.mfft_exec_c2r
        return fn(f._plan, P(src), P(dst), b, flags, None)

    xd = x.cuda()
    yd = torch.empty(shape_out, dtype=dt_out, device="cuda")
    M._check(run(xd, yd, M.DEVICE))
    torch.cuda.synchronize()
    ref = yd.cpu()
    for pinned in (False, True):
        xs = x.pin_memory() if pinned else x
        yh = torch.empty(shape_out, dtype=dt_out, pin_memory=pinned)
        M._check(run(xs, yh, M.HOST))
        assert torch.equal(yh, ref), (kind, n, b, pinned)


@pytest.mark.parametrize("n", [1 << 16, 1 << 17, 1 << 18, 1 << 19, 1 << 20])
def test_tma_fourstep_inverse_odd_batch_in_place(M, n):
    """Four-step sizes whose tiles move by TMA: forward and inverse of an odd
    batch against FP64; in place equal to out of place; one line alone equal
    to the same line inside the batch (bit for bit)."""
    import torch
    b = 3
    x = O.normal_c64((b, n), seed=5000 + n)
    f = M.MetalFFT(n)
    xd = torch.from_numpy(x).cuda()
    y = torch.empty_like(xd)
    f.exec(xd, y, b, M.FORWARD)
    zi = torch.empty_like(xd)
    f.exec(xd, zi, b, M.INVERSE)
    one = torch.empty_like(xd[1:2])
    f.exec(xd[1:2].clone(), one, 1, M.FORWARD)
    ip = xd.clone()
    f.exec(ip, ip, b, M.FORWARD)
    torch.cuda.synchronize()
    assert M.lib.mfft_context_check(M.shared_context()) == 0
    assert O.rel_rms(y.cpu().numpy(), O.truth(x)) < TOL_BIG
    assert O.rel_rms(zi.cpu().numpy(), O.truth(x, inverse=True)) < TOL_BIG
    assert torch.equal(ip, y)
    assert torch.equal(one[0], y[1])


def test_plans_of_the_shared_context_on_concurrent_threads(M):
    # MetalContext.shared is one lock-protected context used by every MetalFFT
    # instance (MetalContext.swift:79-88); each instance is single-threaded
    # (MetalFFT.swift:9).  Here four threads, each with its own plans on the
    # shared context, run host-array calls at the same time (ctypes releases
    # the GIL during each call): the staged chunk pipeline, the single-chunk
    # path, a four-step plan and the tensor-core kernel overlap.  Every result
    # matches FP64 and repeats bitwise.
    import threading
    jobs = [("c2c-chunks", 4096, 1024, 0), ("c2c-small", 1024, 64, 0),
            ("fourstep", 1 << 16, 8, 0), ("tc-split", 4096, 512, M.TC_FP16_SPLIT3)]
    errors, results = [], {}

    def work(name, n, b, tc, seed):
        try:
            f = M.MetalFFT(n)
            rng = np.random.default_rng(seed)
            x = (rng.standard_normal((b, n)) + 1j * rng.standard_normal((b, n))).astype(np.complex64)
            first = None
            for _ in range(4):
                y = f.forward_batch(x, tc_variant=tc)
                if first is None:
                    first = y.copy()
                elif not np.array_equal(y, first):
                    errors.append("%s: a repeated call differs" % name)
            results[name] = (x, first)
        except Exception as e:  # noqa: BLE001 -- reported below
            errors.append("%s: %r" % (name, e))

    threads = [threading.Thread(target=work, args=(name, n, b, tc, 100 + i))
               for i, (name, n, b, tc) in enumerate(jobs)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
    for name, n, b, tc in jobs:
        x, y = results[name]
        ref = np.fft.fft(x.astype(np.complex128), axis=-1)
        err = float(np.linalg.norm(y - ref) / np.linalg.norm(ref))
        assert err <= (3e-6 if tc or n > 16384 else 2e-6), (name, err)
