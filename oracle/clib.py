"""ctypes access to the oracle's C libraries (test infrastructure only).

  restatement()  _build/liboracle.so: C restatements (ref_fft.c, kfft_fp32.c)
  reference()    _ref/libref.so: the reference's own reference.cpp compiled from its sources
                 (None when it was never built, e.g. without the reference checkout)
Row helpers take numpy float32 arrays and loop over rows in C; calls release the GIL, so
callers may spread rows over threads.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_rest = None
_ref = None


def restatement():
    global _rest
    if _rest is None:
        lib = C.CDLL(str(HERE / "_build" / "liboracle.so"))
        for name in ("orc_ref_fft", "orc_ref_r2c", "orc_ref_c2r", "orc_kfft_r2c", "orc_kfft_c2r"):
            getattr(lib, name).argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
            getattr(lib, name).restype = None
        lib.orc_kfft_fwd.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int]
        lib.orc_kfft_fwd.restype = None
        lib.orc_plane_k.argtypes = [C.c_uint32]
        lib.orc_plane_k.restype = C.c_uint32
        lib.orc_max_rel_scaled.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        lib.orc_max_rel_scaled.restype = C.c_double
        lib.orc_pattern_at.argtypes = [C.c_size_t]
        lib.orc_pattern_at.restype = C.c_float
        _rest = lib
    return _rest


def reference():
    global _ref
    if _ref is None:
        path = HERE / "_ref" / "libref.so"
        if not path.exists():
            return None
        lib = C.CDLL(str(path))
        for name in ("ref_fft_rows", "ref_r2c_rows", "ref_c2r_rows"):
            getattr(lib, name).argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]
            getattr(lib, name).restype = None
        lib.ref_max_rel_scaled.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        lib.ref_max_rel_scaled.restype = C.c_double
        lib.ref_pattern_at.argtypes = [C.c_size_t]
        lib.ref_pattern_at.restype = C.c_float
        _ref = lib
    return _ref


def _rows(fn, x: np.ndarray, n: int, in_w: int, out_w: int, extra=()):
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, in_w)
    out = np.empty((x.shape[0], out_w), np.float32)
    for r in range(x.shape[0]):
        fn(x[r].ctypes.data, out[r].ctypes.data, n, *extra)
    return out


def rest_fft(x, n):
    return _rows(restatement().orc_ref_fft, x, n, 2 * n, 2 * n)


def rest_r2c(x, n):
    return _rows(restatement().orc_ref_r2c, x, n, n, n + 2)


def rest_c2r(x, n):
    return _rows(restatement().orc_ref_c2r, x, n, n + 2, n)


def kfft_fwd(x, n, sign=-1):
    return _rows(restatement().orc_kfft_fwd, x, n, 2 * n, 2 * n, (sign,))


def kfft_r2c(x, n):
    return _rows(restatement().orc_kfft_r2c, x, n, n, n + 2)


def kfft_c2r(x, n):
    return _rows(restatement().orc_kfft_c2r, x, n, n + 2, n)


def ref_fft(x, n):
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 2 * n)
    out = np.empty_like(x)
    reference().ref_fft_rows(x.ctypes.data, out.ctypes.data, n, x.shape[0])
    return out


def ref_r2c(x, n):
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, n)
    out = np.empty((x.shape[0], n + 2), np.float32)
    reference().ref_r2c_rows(x.ctypes.data, out.ctypes.data, n, x.shape[0])
    return out


def ref_c2r(x, n):
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, n + 2)
    out = np.empty((x.shape[0], n), np.float32)
    reference().ref_c2r_rows(x.ctypes.data, out.ctypes.data, n, x.shape[0])
    return out
