"""Failure path on the GPU without a fault: a bounded device-side wait that
can never be satisfied gives up after its limit, the host call reports
FFTError.timeout, and the context keeps working."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import metalfft_b200
    return metalfft_b200


def test_bounded_wait_expires_and_context_survives(M):
    import time
    ctx = M.shared_context()
    t0 = time.perf_counter()
    st = M.lib.mfft_selftest_bounded_wait(ctx, 20_000_000)  # 20 ms limit
    dt = time.perf_counter() - t0
    assert st == 11, M.lib.mfft_status_string(st)  # MFFT_ERR_TIMEOUT
    assert 0.015 < dt < 5.0
    # the error word was read and cleared; nothing else is pending
    assert M.lib.mfft_context_check(ctx) == 0
    # the context still runs transforms correctly
    x = O.uniform_c64((16, 4096), seed=99)
    y = M.MetalFFT(4096).forward_batch(x)
    assert O.rel_rms(y, O.truth(x)) < 2e-6


def test_selftest_rejects_bad_limits(M):
    ctx = M.shared_context()
    assert M.lib.mfft_selftest_bounded_wait(ctx, 10) == 10
    assert M.lib.mfft_selftest_bounded_wait(ctx, 10 ** 10) == 10
    assert M.lib.mfft_selftest_bounded_wait(None, 1_000_000) == 10
