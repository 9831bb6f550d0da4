"""mfft_fourstep_noalloc: the four-step FFT for callers that cannot allocate
device memory (an external allocator owns the device, a real-time host
reserves memory once at start-up, a plug-in host forbids allocation).  Its
intermediate is a fixed 16 MiB device array shared by every call, so calls in
a row must each give the same result as the allocating entry point
(mfft_exec_c2c on a plan) and as the FP64 oracle, within the four-step
tolerance of the other tests.

Every size it takes (2^15 .. 2^20: even splits 256 x 256 ... 1024 x 1024 and
uneven ones 128 x 256, 256 x 512, 512 x 1024) runs forward and inverse, with
batch = 2^21 / n + 1 lines so that each call goes through the array in one
full chunk and one partial chunk.
This file is collected last, so a stop-at-first-failure run has already run
every other test when it starts."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

TOL_BIG = 3e-6  # four-step sizes, as tests/test_fft_gpu.py
SCRATCH_POINTS = 1 << 21
BIG = [1 << 15, 1 << 16, 1 << 17, 1 << 18, 1 << 19, 1 << 20]


def test_noalloc_rejects_sizes_outside_its_range():
    from metalfft_b200 import _lib
    lib = _lib.load()
    for n in [4096, 1 << 21, 3 << 15]:
        st = lib.mfft_fourstep_noalloc(None, None, n, 1, -1, None)
        assert st == 8  # MFFT_ERR_UNSUPPORTED_SIZE
        buf = ctypes.create_string_buffer(256)
        lib.mfft_last_error(buf, 256)
        assert b"32768 to 1048576" in buf.value


def _noalloc(M, x, out, n, batch, direction):
    import torch
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return M.lib.mfft_fourstep_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                       n, batch, direction, stream)


@pytest.mark.gpu
@pytest.mark.parametrize("n", BIG)
def test_noalloc_every_size_both_directions_two_calls_in_a_row(n):
    import torch

    import metalfft_b200 as M
    batch = SCRATCH_POINTS // n + 1  # one full chunk of the array, then one line
    for k, direction in enumerate([M.FORWARD, M.INVERSE]):
        xh = O.normal_c64((batch, n), seed=7000 + 2 * n + k)
        x = torch.from_numpy(xh).cuda()
        ref = torch.empty_like(x)
        M.MetalFFT(n).exec(x, ref, batch, direction)
        truth = O.truth(xh, inverse=(direction == M.INVERSE))
        outs = []
        for _ in range(2):  # the second call starts from the array the first one left
            out = torch.full_like(x, float("nan"))
            assert _noalloc(M, x, out, n, batch, direction) == 0
            torch.cuda.synchronize()
            outs.append(out)
        for out in outs:
            err_alloc = float(torch.linalg.vector_norm(out - ref) / torch.linalg.vector_norm(ref))
            assert np.isfinite(err_alloc) and err_alloc < TOL_BIG, (n, batch, direction, err_alloc)
            yh = out.cpu().numpy()
            err_fp64 = O.rel_rms(yh, truth)
            assert err_fp64 < TOL_BIG, (n, batch, direction, err_fp64)
            # the last, partial chunk (one line) on its own
            assert O.rel_rms(yh[-1:], truth[-1:]) < TOL_BIG, (n, direction)
        assert torch.equal(outs[0], outs[1])


@pytest.mark.gpu
def test_noalloc_in_place():
    import torch

    import metalfft_b200 as M
    n, batch = 1 << 17, 5
    xh = O.normal_c64((batch, n), seed=7100)
    x = torch.from_numpy(xh).cuda()
    assert _noalloc(M, x, x, n, batch, M.FORWARD) == 0
    torch.cuda.synchronize()
    assert O.rel_rms(x.cpu().numpy(), O.truth(xh)) < TOL_BIG
