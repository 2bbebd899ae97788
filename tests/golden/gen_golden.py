"""Generate tests/golden/ref_oracle_vectors.npz from the reference's own FP64 oracle.

The reference (TruNcat3/ascend-fft) ships no golden output vectors; its results are pinned by
its FP64 oracle src/framework/reference.cpp.  This script runs that oracle, compiled from the
reference's sources into oracle/_ref/libref.so by `make -C oracle`, on deterministic inputs
and stores inputs and outputs:

  c2c_<n>    patternAt input (reference.cpp:10-12) and the "sin" harness input
             (src/host/fft_check.cpp genC2CInput), batch 2, n in 64..4096, plus 8192 for r2c
  r2c_<n>    patternAt real rows (tests/test_framework.cpp:24-26), n in 128..8192
  c2r_<n>    patternAt half spectra with Nyquist imaginary 0 (test_framework.cpp:104-106)
  mrs        maxRelScaled cases of tests/test_runtime_guards.cpp:64-85

    make -C oracle && python tests/golden/gen_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import clib  # noqa: E402
from oracle import fft_oracle as O  # noqa: E402


def main():
    ref = clib.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libref.so missing: run `make -C oracle` with the reference present")
    out = {}
    for n in [64, 128, 256, 512, 1024, 2048, 4096]:
        pat = np.stack([O.pattern_at(np.arange(2 * n) + r * 2 * n) for r in range(2)])
        sin = O.harness_input("sin", n, 2)
        for tag, x in (("pattern", pat), ("sin", sin)):
            out[f"c2c_{tag}_{n}_in"] = x
            out[f"c2c_{tag}_{n}_out"] = clib.ref_fft(x, n)
    for n in [128, 256, 512, 1024, 2048, 4096, 8192]:
        x = np.stack([O.pattern_at(np.arange(n) + r * n) for r in range(2)])
        out[f"r2c_{n}_in"] = x
        out[f"r2c_{n}_out"] = clib.ref_r2c(x, n)
    for n in [64, 128, 256, 512, 1024, 2048, 4096]:
        h = np.stack([O.pattern_at(np.arange(n + 2) + r * (n + 2)) for r in range(2)])
        h[:, n + 1] = 0.0
        out[f"c2r_{n}_in"] = h
        out[f"c2r_{n}_out"] = clib.ref_c2r(h, n)
    cases = np.array([[1, 0, 0, 0], [1e-6, 0, 0, 0], [1e-6, 0, 1e-8, 0], [101, 0, 100, 0]], np.float32)
    out["mrs_cases"] = cases
    out["mrs_values"] = np.array([ref.ref_max_rel_scaled(c[:2].ctypes.data, c[2:].ctypes.data, 2)
                                  for c in cases])
    path = Path(__file__).resolve().parent / "ref_oracle_vectors.npz"
    np.savez_compressed(path, **out)
    print(path, sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
