"""CPU checks of the C ABI: the built library loads, exports every entry point include/*.h
declares, and its pure-host helpers behave like the reference's (no GPU calls)."""
import math
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"\b(bfly_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    import bfly
    return bfly.load()


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s


def test_python_signatures_cover_header():
    from bfly import _lib
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_version(lib):
    assert b"sm_100a" in lib.bfly_version()


def test_max_rel_scaled_semantics(lib):
    """Same cases as the reference's tests/test_runtime_guards.cpp:64-85."""
    def mrs(got, ref):
        g = np.asarray(got, np.float32)
        r = np.asarray(ref, np.float32)
        return lib.bfly_max_rel_scaled(g.ctypes.data, r.ctypes.data, len(g))
    assert mrs([1.0, 0.0], [0.0, 0.0]) == 1.0
    assert mrs([1e-6, 0.0], [0.0, 0.0]) > 0
    assert mrs([1e-6, 0.0], [1e-8, 0.0]) < 1e-4
    for v in (math.nan, math.inf, -math.inf):
        assert math.isinf(mrs([v, 0.0], [1e-8, 0.0]))
        assert math.isinf(mrs([0.0, 0.0], [v, 0.0]))
    assert math.isinf(lib.bfly_max_rel_scaled(None, np.zeros(2, np.float32).ctypes.data, 2))
    assert lib.bfly_max_rel_scaled(None, None, 0) == 0
    assert mrs([101.0, 0.0], [100.0, 0.0]) == pytest.approx(0.01)


def test_pattern_and_sampling_match_oracle(lib):
    import oracle.fft_oracle as O
    idx = np.arange(5000)
    ours = np.array([lib.bfly_pattern_at(int(i)) for i in idx], np.float32)
    assert np.array_equal(ours, O.pattern_at(idx))
    import ctypes
    for batch, want in ((0, 8), (1, 8), (5, 8), (8, 8), (1000, 8), (1000, 1), (3, 0)):
        buf = (ctypes.c_uint32 * 16)()
        cnt = lib.bfly_sample_batches(batch, want, buf, 16)
        assert list(buf[:cnt]) == O.sample_batches(batch, want)


def test_noalloc_long_size_guard_without_gpu(lib):
    """The allocation-free long C2C rejects oversize requests before any CUDA call, including a
    batch whose product with n wraps in 64 bits (65536 * (2^48 + 1) = 65536 mod 2^64)."""
    import ctypes as C
    p = C.c_void_p(16)   # never dereferenced: every call is rejected first
    f = lib.bfly_exec_c2c_long_noalloc
    assert f(p, p, 65536, (1 << 48) + 1, -1, 1.0, None) == -12
    assert f(p, p, 65536, 65, -1, 1.0, None) == -12
    assert f(p, p, 8192, 513, 1, 1.0, None) == -12
    assert f(p, p, 8192, 0, -1, 1.0, None) == -8
    assert f(None, p, 8192, 1, -1, 1.0, None) == -10
