"""ctypes binding of libmfft.so (the C ABI declared in include/mfft.h).

The shared library is built in-tree by ``__graft_entry__.build()`` (make in
metalfft_b200/csrc).  There is no fallback: importing the package without the
library raises ImportError, and every call returns the library's own status.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmfft.so")

c_int, c_int64, c_double, c_void_p, c_char_p, c_size_t = (
    ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p,
    ctypes.c_size_t)
P = ctypes.POINTER

# (name, restype, argtypes) for every entry point of include/mfft.h
SIGNATURES = [
    ("mfft_status_string", c_char_p, [c_int]),
    ("mfft_last_error", c_int, [c_char_p, c_size_t]),
    ("mfft_last_error_detail", c_int, [P(c_int64), P(c_int64), P(c_int64)]),
    ("mfft_context_shared", c_int, [P(c_void_p)]),
    ("mfft_context_create", c_int, [c_int, P(c_void_p)]),
    ("mfft_context_destroy", c_int, [c_void_p]),
    ("mfft_context_sm_count", c_int, [c_void_p]),
    ("mfft_context_check", c_int, [c_void_p]),
    ("mfft_selftest_bounded_wait", c_int, [c_void_p, c_int64]),
    ("mfft_plan_create", c_int, [c_void_p, c_int64, P(c_void_p)]),
    ("mfft_plan_destroy", c_int, [c_void_p]),
    ("mfft_plan_size", c_int64, [c_void_p]),
    ("mfft_recommended_fft_size", c_int64, [c_int64]),
    ("mfft_autotune", c_int, [c_void_p, c_int64, c_int64, P(c_int), P(c_int), P(c_int)]),
    ("mfft_plan_kernel_info", c_int, [c_void_p, P(c_int), P(c_int), P(c_int), P(c_int)]),
    ("mfft_plan_set_kernel", c_int, [c_void_p, c_int, c_int, c_int]),
    ("mfft_list_kernels", c_int, [c_int64, P(c_int), P(c_int), P(c_int), c_int]),
    ("mfft_autotune_fourstep", c_int, [c_void_p, c_int64, P(c_int)]),
    ("mfft_plan_set_split", c_int, [c_void_p, c_int64]),
    ("mfft_plan_split", c_int, [c_void_p, P(c_int64), P(c_int64)]),
    ("mfft_list_splits", c_int, [c_int64, P(c_int64), c_int]),
    ("mfft_exec_c2c", c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int, c_void_p]),
    ("mfft_exec_c2c_backward", c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int, c_void_p]),
    ("mfft_exec_c2c_tc", c_int,
     [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int, c_int, c_void_p]),
    ("mfft_exec_r2c", c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_void_p]),
    ("mfft_exec_c2r", c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_void_p]),
    ("mfft_fourstep_noalloc", c_int, [c_void_p, c_void_p, c_int64, c_int64, c_int, c_void_p]),
    ("mfft_multi_create", c_int, [c_void_p, c_void_p, c_int, P(c_void_p)]),
    ("mfft_multi_destroy", c_int, [c_void_p]),
    ("mfft_multi_points", c_int64, [c_void_p]),
    ("mfft_multi_exec", c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]),
    ("mfft_conv_create", c_int, [c_void_p, c_void_p, c_int64, c_int64, P(c_void_p)]),
    ("mfft_conv_destroy", c_int, [c_void_p]),
    ("mfft_conv_block_size", c_int64, [c_void_p]),
    ("mfft_conv_hop_size", c_int64, [c_void_p]),
    ("mfft_conv_set_precision", c_int, [c_void_p, c_int]),
    ("mfft_conv_kernel_len", c_int64, [c_void_p]),
    ("mfft_conv_apply", c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int, c_void_p]),
    ("mfft_conv_backward", c_int,
     [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    ("mfft_corr_create", c_int, [c_void_p, c_int64, P(c_void_p)]),
    ("mfft_corr_destroy", c_int, [c_void_p]),
    ("mfft_corr_cross", c_int,
     [c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int, c_void_p]),
    ("mfft_window", c_int, [c_int, c_int64, c_double, c_void_p]),
    ("mfft_analyzer_create", c_int,
     [c_void_p, c_int64, c_double, c_int, c_double, P(c_void_p)]),
    ("mfft_analyzer_destroy", c_int, [c_void_p]),
    ("mfft_spectral_create", c_int, [c_void_p, c_int64, c_int64, c_int, c_double, P(c_void_p)]),
    ("mfft_spectral_destroy", c_int, [c_void_p]),
    ("mfft_stft_frame_count", c_int64, [c_void_p, c_int64]),
    ("mfft_stft_analyze", c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_int, c_void_p]),
    ("mfft_psd_welch", c_int, [c_void_p, c_void_p, c_int64, c_double, c_void_p, c_int, c_void_p]),
    ("mfft_psd_coherence", c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int, c_void_p]),
    ("mfft_psd_cross_spectral", c_int,
     [c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]),
    ("mfft_analyzer_analyze", c_int,
     [c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int, c_void_p]),
    ("mfft_sar_default_params", c_int, [c_int64, c_int64, c_int64, c_double, c_void_p]),
    ("mfft_sar_chirp_reference", c_int, [c_void_p, c_void_p]),
    ("mfft_sar_simulate", c_int, [c_void_p, c_void_p, c_void_p, c_int, c_double, ctypes.c_uint64, c_void_p,
                                  c_void_p]),
    ("mfft_sar_quantize", c_int, [c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("mfft_sar_create", c_int, [c_void_p, c_void_p, c_void_p, P(c_void_p)]),
    ("mfft_sar_destroy", c_int, [c_void_p]),
    ("mfft_sar_forward", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("mfft_sar_set_intermediate", c_int, [c_void_p, c_int]),
    ("mfft_sar_backward_phase", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("mfft_sar_step_graph", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p]),
    ("mfft_sar_focus", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
]

_lib = None
_lock = threading.Lock()


def load():
    """Load libmfft.so once and declare every signature; raise if absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "libmfft.so is not built (expected at %s); run __graft_entry__.build()" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def exported_symbols():
    return [name for name, _, _ in SIGNATURES]
