"""ctypes binding of libbfly_b200.so (the C ABI declared in include/bfly_b200.h).

The shared library is built in-tree by ascend-fft_b200/build.py.  Loading fails loudly when it
is missing: there is no CPU fallback for any transform.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libbfly_b200.so"

c_ctx = C.c_void_p
c_plan = C.c_void_p

# name -> (restype, argtypes); every symbol declared in include/bfly_b200.h
SIGNATURES = {
    "bfly_version": (C.c_char_p, []),
    "bfly_context_create": (C.c_int, [C.POINTER(c_ctx)]),
    "bfly_context_destroy": (None, [c_ctx]),
    "bfly_context_init": (C.c_int, [c_ctx, C.c_char_p, C.c_char_p, C.c_char_p]),
    "bfly_context_init_device": (C.c_int, [c_ctx, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]),
    "bfly_context_enumerate": (C.c_int, [c_ctx, C.c_uint32, C.c_uint32, C.c_char_p, C.c_size_t,
                                         C.POINTER(C.c_int), C.POINTER(C.c_size_t)]),
    "bfly_context_select": (C.c_int, [c_ctx, C.c_uint32, C.c_uint32, C.c_int, C.POINTER(c_plan),
                                      C.c_char_p, C.c_size_t]),
    "bfly_context_make_plan": (C.c_int, [c_ctx, C.c_uint32, C.c_uint32, C.c_char_p,
                                         C.POINTER(c_plan)]),
    "bfly_context_set_tuning_cache": (C.c_int, [c_ctx, C.c_char_p]),
    "bfly_context_stream": (C.c_void_p, [c_ctx]),
    "bfly_plan_destroy": (None, [c_plan]),
    "bfly_plan_candidate_id": (C.c_int, [c_plan, C.c_char_p, C.c_size_t]),
    "bfly_plan_prepare": (C.c_int, [c_plan, C.c_uint32, C.c_uint32]),
    "bfly_plan_run_c2c": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "bfly_plan_run_c2c_many": (C.c_int, [c_plan, C.c_void_p, C.c_size_t]),
    "bfly_plan_run_r2c": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "bfly_plan_run_c2r": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "bfly_plan_measure": (C.c_int, [c_plan, C.c_uint32, C.c_uint32, C.c_void_p]),
    "bfly_plan_run_c2c_inverse": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32,
                                            C.c_uint32, C.c_float]),
    "bfly_plan_run_c2c_long": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                         C.c_int]),
    "bfly_plan_exec_c2c_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                           C.c_int, C.c_float, C.c_void_p]),
    "bfly_plan_exec_c2c_2d_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                              C.c_uint64, C.c_int, C.c_float, C.c_void_p]),
    "bfly_plan_exec_r2c_2d_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                              C.c_uint64, C.c_float, C.c_void_p]),
    "bfly_plan_exec_c2r_2d_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                              C.c_uint64, C.c_float, C.c_void_p]),
    "bfly_plan_exec_c2c_axis_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                                C.c_uint64, C.c_int, C.c_float, C.c_void_p]),
    "bfly_plan_exec_stft_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                            C.c_uint64, C.c_uint32, C.c_int, C.c_void_p,
                                            C.POINTER(C.c_uint64), C.c_void_p]),
    "bfly_plan_exec_istft_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                             C.c_uint32, C.c_uint32, C.c_int, C.c_void_p, C.c_uint64,
                                             C.c_float, C.c_void_p]),
    "bfly_plan_exec_stft_backward_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                                     C.c_uint64, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p]),
    "bfly_plan_exec_istft_backward_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                                      C.c_uint32, C.c_uint32, C.c_int, C.c_void_p, C.c_uint64,
                                                      C.c_float, C.c_void_p]),
    "bfly_plan_exec_r2c_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                           C.c_float, C.c_float, C.c_void_p]),
    "bfly_plan_exec_c2r_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                           C.c_float, C.c_float, C.c_float, C.c_void_p]),
    "bfly_plan_exec_c2c_tc_async": (C.c_int, [c_plan, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                              C.c_int, C.c_float, C.c_int, C.c_void_p]),
    "bfly_tc_device_status": (C.c_int, [C.POINTER(C.c_uint)]),
    "bfly_long_device_status": (C.c_int, [C.POINTER(C.c_uint)]),
    "bfly_ragged_create": (C.c_int, [c_plan, C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p)]),
    "bfly_ragged_exec_async": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bfly_ragged_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]),
    "bfly_ragged_device_status": (C.c_int, [C.POINTER(C.c_uint)]),
    "bfly_ragged_destroy": (None, [C.c_void_p]),
    "bfly_ragged_create_config": (C.c_int, [c_plan, C.c_void_p, C.c_size_t, C.c_int, C.c_uint32,
                                            C.POINTER(C.c_void_p)]),
    "bfly_context_tune_ragged": (C.c_int, [C.c_void_p, c_plan, C.c_void_p, C.c_size_t,
                                           C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "bfly_ragged_config": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint32)]),
    "bfly_exec_c2c_long_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                             C.c_int, C.c_float, C.c_void_p]),
    "bfly_max_rel_scaled": (C.c_double, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "bfly_pattern_at": (C.c_float, [C.c_size_t]),
    "bfly_sample_batches": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32]),
}


class RaggedRequest(C.Structure):
    """bfly_ragged_request of include/bfly_b200.h."""
    _fields_ = [("d_in", C.c_void_p), ("d_out", C.c_void_p), ("n", C.c_uint32),
                ("direction", C.c_int32), ("batch", C.c_uint64), ("scale", C.c_float),
                ("reserved", C.c_uint32)]


class HostRequest(C.Structure):
    """bfly_host_request of include/bfly_b200.h."""
    _fields_ = [("in_", C.c_void_p), ("out", C.c_void_p), ("n", C.c_uint32), ("batch", C.c_uint32),
                ("direction", C.c_int32), ("scale", C.c_float)]


class Metric(C.Structure):
    _fields_ = [("eta_us", C.c_double), ("measured_us", C.c_double),
                ("max_rel_err", C.c_double), ("measured_ok", C.c_int)]


_lib = None


def load() -> C.CDLL:
    """Load and declare the library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python ascend-fft_b200/build.py` "
                          "(the library has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
