"""mfft_fourstep_noalloc: the four-step FFT for callers that cannot allocate
device memory (an external allocator owns the device, a real-time host
reserves memory once at start-up, a plug-in host forbids allocation).  Its
intermediate is a fixed 16 MiB device array shared by every call, so two
calls in a row must each give the same result as the allocating entry point
(mfft_exec_c2c on a plan), within the four-step tolerance of the other tests.
This file is collected last, so a stop-at-first-failure run has already run
every other test when it starts."""
import ctypes

import numpy as np
import pytest

TOL_BIG = 3e-6  # four-step sizes, as tests/test_fft_gpu.py


def test_noalloc_rejects_sizes_outside_its_range():
    from metalfft_b200 import _lib
    lib = _lib.load()
    for n in [4096, 1 << 21, 3 << 15]:
        st = lib.mfft_fourstep_noalloc(None, None, n, 1, -1, None)
        assert st == 8  # MFFT_ERR_UNSUPPORTED_SIZE
        buf = ctypes.create_string_buffer(256)
        lib.mfft_last_error(buf, 256)
        assert b"32768 to 1048576" in buf.value


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_two_calls_in_a_row():
    import torch

    import metalfft_b200 as M
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(1234)
    # first: 2^20 x 3 lines forward (two chunks through the 16 MiB array);
    # second: 2^16 x 5 lines inverse, reusing the array the first call left.
    for n, batch, direction in [(1 << 20, 3, M.FORWARD), (1 << 16, 5, M.INVERSE)]:
        x = torch.randn(batch, n, dtype=torch.complex64, device="cuda", generator=g)
        ref = torch.empty_like(x)
        M.MetalFFT(n).exec(x, ref, batch, direction)
        out = torch.full_like(x, float("nan"))
        st = M.lib.mfft_fourstep_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                         n, batch, direction, stream)
        assert st == 0
        torch.cuda.synchronize()
        err = float(torch.linalg.vector_norm(out - ref) / torch.linalg.vector_norm(ref))
        assert np.isfinite(err) and err < TOL_BIG, (n, batch, direction, err)
