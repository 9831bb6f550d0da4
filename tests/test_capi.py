"""The C ABI library loads and exports every entry point include/mfft.h
declares, and its host-only logic works without a GPU (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mfft.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(mfft_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["mfft_plan_create", "mfft_exec_c2c", "mfft_exec_c2c_tc", "mfft_multi_exec",
                 "mfft_conv_apply", "mfft_conv_backward", "mfft_corr_cross",
                 "mfft_analyzer_analyze", "mfft_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from metalfft_b200 import _lib
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares a signature for each of them
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_status_strings_and_host_helpers():
    from metalfft_b200 import _lib
    lib = _lib.load()
    assert lib.mfft_status_string(0) == b"success"
    assert b"Unsupported FFT size" in lib.mfft_status_string(8)
    # Convolver.recommendedFFTSize(forKernelCount:) (Convolve.swift:83-86)
    assert lib.mfft_recommended_fft_size(100) == 128
    assert lib.mfft_recommended_fft_size(128) == 256
    assert lib.mfft_recommended_fft_size(16384) == 0


def test_four_step_split_lists():
    """Admissible splits n = n1 x n2 (64 <= n1 <= 1024, 128 <= n2 <= 1024) of
    the four-step sizes; none below 32768."""
    from metalfft_b200 import _lib
    lib = _lib.load()
    buf = (ctypes.c_int64 * 8)()
    want = {1 << 15: [64, 128, 256], 1 << 16: [64, 128, 256, 512], 1 << 17: [128, 256, 512, 1024],
            1 << 18: [256, 512, 1024], 1 << 19: [512, 1024], 1 << 20: [1024]}
    for n, w in want.items():
        m = lib.mfft_list_splits(n, buf, 8)
        assert list(buf[:m]) == w, n
    for n in (4096, 16384, 1 << 21, 3 << 15):
        assert lib.mfft_list_splits(n, buf, 8) == 0
    assert lib.mfft_list_splits(1 << 16, buf, 2) == 4  # count beyond cap


def test_no_device_is_reported_not_faked():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from metalfft_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.mfft_context_shared(ctypes.byref(h))
    assert st == 1  # MFFT_ERR_NO_DEVICE == FFTError.noMetalDevice
    buf = ctypes.create_string_buffer(256)
    assert lib.mfft_last_error(buf, 256) == 1
    assert b"No CUDA device" in buf.value


def test_window_coefficients_match_oracle():
    import numpy as np

    from metalfft_b200 import _lib
    from oracle import oracle as O
    lib = _lib.load()
    for kind in range(6):
        for n in [8, 64, 1024]:
            w = np.empty(n, np.float32)
            assert lib.mfft_window(kind, n, 6.0, w.ctypes.data) == 0
            assert np.max(np.abs(w - O.window(kind, n, 6.0))) < 1e-6
    assert lib.mfft_window(9, 8, 0.0, w.ctypes.data) == 10
