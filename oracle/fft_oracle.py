"""FP64 oracle for the batched FFT (test infrastructure only; see oracle/__init__.py).

Transforms are numpy.fft (pocketfft) on float64/complex128, the oracle the reference's
harness and stdlib baseline use (scripts/bench_stdlib.py:28-68), with the reference's
conventions:
  c2c     X[k] = sum_j x[j] exp(-2 pi i j k / n), unnormalised   (docs/user-guide/transforms.md:22)
  r2c     numpy.fft.rfft, dense [n/2+1] half spectrum            (include/butterfly/plan.hpp:38-40)
  c2r     numpy.fft.irfft incl. 1/n; imaginary parts of bins 0 and n/2 ignored
          (src/framework/reference.cpp:64-79 takes the real part of the mirrored spectrum)
Layouts are interleaved fp32 [batch][2n] / [batch][n+2] as in the reference.
"""
from __future__ import annotations

import math

import numpy as np

# ------------------------------------------------------------------ layout helpers


def to_complex(a: np.ndarray) -> np.ndarray:
    """Interleaved float32 [..., 2m] -> complex128 [..., m]."""
    a = np.asarray(a, dtype=np.float64)
    return a[..., 0::2] + 1j * a[..., 1::2]


def to_interleaved(z: np.ndarray) -> np.ndarray:
    """complex [..., m] -> interleaved float32 [..., 2m] (rounded once)."""
    out = np.empty(z.shape[:-1] + (2 * z.shape[-1],), dtype=np.float32)
    out[..., 0::2] = z.real
    out[..., 1::2] = z.imag
    return out


# ------------------------------------------------------------------ transforms (float64)


def c2c(x: np.ndarray) -> np.ndarray:
    """Forward C2C of interleaved rows [batch][2n] -> complex128 [batch][n]."""
    return np.fft.fft(to_complex(x), axis=-1)


def c2c_inverse(x: np.ndarray, scale: float = 1.0) -> np.ndarray:
    """Unnormalised inverse C2C times scale."""
    z = to_complex(x)
    return np.fft.ifft(z, axis=-1) * (z.shape[-1] * scale)


def r2c(x: np.ndarray) -> np.ndarray:
    """Real rows [batch][n] -> complex128 [batch][n/2+1]."""
    return np.fft.rfft(np.asarray(x, dtype=np.float64), axis=-1)


def c2r(x: np.ndarray, n: int) -> np.ndarray:
    """Half-spectrum rows [batch][n+2] interleaved -> float64 [batch][n], incl. 1/n."""
    return np.fft.irfft(to_complex(x), n=n, axis=-1)


# ------------------------------------------------------------------ metrics


def rel_l2(got: np.ndarray, ref: np.ndarray) -> float:
    """||got - ref||_2 / ||ref||_2 over the whole array (complex or real)."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    if np.iscomplexobj(ref) and not np.iscomplexobj(got):
        got = to_complex(got)
    num = np.linalg.norm((got.astype(np.complex128) - ref).ravel())
    den = np.linalg.norm(ref.ravel())
    return float(num / den) if den > 0 else float(num)


def rel_l2_rows(got: np.ndarray, ref: np.ndarray) -> float:
    """Maximum over rows of the per-row relative L2 error."""
    got = np.asarray(got)
    if np.iscomplexobj(ref) and not np.iscomplexobj(got):
        got = to_complex(got)
    d = np.linalg.norm(got.astype(np.complex128) - ref, axis=-1)
    r = np.linalg.norm(ref, axis=-1)
    r = np.where(r > 0, r, 1.0)
    return float((d / r).max()) if d.size else 0.0


def max_rel_scaled(got: np.ndarray, ref: np.ndarray) -> float:
    """The reference's acceptance metric max|got-ref| / max(1, max|ref|) over float
    components, infinity for non-finite values (include/butterfly/reference.hpp:30-41)."""
    g = np.asarray(got, dtype=np.float64).ravel()
    r = np.asarray(ref, dtype=np.float64).ravel()
    if g.size == 0:
        return 0.0
    if not (np.all(np.isfinite(g)) and np.all(np.isfinite(r))):
        return math.inf
    return float(np.abs(g - r).max() / max(1.0, np.abs(r).max()))


def max_rel_scaled_rows(got: np.ndarray, ref: np.ndarray) -> float:
    """Worst per-row maxRelScaled, the way the reference's harness gates every row."""
    g = np.asarray(got, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    if not (np.all(np.isfinite(g)) and np.all(np.isfinite(r))):
        return math.inf
    err = np.abs(g - r).max(axis=-1)
    scale = np.maximum(1.0, np.abs(r).max(axis=-1))
    return float((err / scale).max()) if err.size else 0.0


# ------------------------------------------------------------------ reference helpers


def pattern_at(i: np.ndarray) -> np.ndarray:
    """((i * 2654435761) mod 2^32 mod 1000) / 1000 - 0.5 in float32 (reference.cpp:10-12)."""
    i = np.asarray(i, dtype=np.uint64)
    h = (i * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)
    return ((h % np.uint64(1000)).astype(np.float32) / np.float32(1000.0) - np.float32(0.5)).astype(np.float32)


def sample_batches(batch: int, want: int = 8) -> list[int]:
    """Evenly spread row indices including 0 and batch-1 (reference.hpp:48-60)."""
    if batch == 0 or want == 0:
        return []
    if batch <= want:
        return list(range(batch))
    if want == 1:
        return [0]
    return [i * (batch - 1) // (want - 1) for i in range(want)]


def app_hash(b: np.ndarray, k: np.ndarray) -> np.ndarray:
    """xorshift32 mix of the reference harness (src/host/fft_check.cpp:63-69)."""
    b = np.asarray(b, dtype=np.uint64)
    k = np.asarray(k, dtype=np.uint64)
    m = np.uint64(0xFFFFFFFF)
    x = (b * np.uint64(2654435761) + k * np.uint64(40503)) & m
    for _ in range(2):
        x ^= (x << np.uint64(13)) & m
        x ^= x >> np.uint64(17)
        x ^= (x << np.uint64(5)) & m
    return x.astype(np.uint32)


def harness_input(mode: str, n: int, batch: int, seed: int = 0) -> np.ndarray:
    """Deterministic C2C inputs of the reference harness (fft_check.cpp:70-192), interleaved
    float32 [batch][2n].  Modes: sin, zero, impulse, constant, tone, alternating, random,
    dynamic, near-cancellation, ofdm, radar, dl."""
    b = np.arange(batch, dtype=np.uint64)[:, None]
    k = np.arange(n, dtype=np.uint64)[None, :]
    re = np.zeros((batch, n), np.float32)
    im = np.zeros((batch, n), np.float32)
    if mode in ("sin", "deterministic-sin-cos"):
        i = np.arange(2 * n * batch, dtype=np.float64)
        return (np.sin(0.011 * i) + 0.25 * np.cos(0.037 * i)).astype(np.float32).reshape(batch, 2 * n)
    if mode == "impulse":
        re = (k == (b % np.uint64(n))).astype(np.float32)
    elif mode == "constant":
        re[:] = 0.25
        im[:] = -0.5
    elif mode in ("tone", "single-tone"):
        tone = (1 + (b % np.uint64(7))).astype(np.float64)
        ph = 2.0 * np.pi * tone * k.astype(np.float64) / n
        re = np.cos(ph).astype(np.float32)
        im = np.sin(ph).astype(np.float32)
    elif mode in ("alternating", "nyquist-alternating"):
        re = np.where(k & np.uint64(1), -1.0, 1.0).astype(np.float32) * np.ones((batch, 1), np.float32)
    elif mode in ("random", "random-seeded"):
        bs = b ^ np.uint64(seed)
        x1 = app_hash(bs, k).astype(np.int64)
        x2 = app_hash(bs, k ^ np.uint64(0x9E37)).astype(np.int64)
        re = ((x1 & 0xFFFF) - 32768).astype(np.float32) * np.float32(1.0 / 32768.0)
        im = ((x2 & 0xFFFF) - 32768).astype(np.float32) * np.float32(1.0 / 32768.0)
    elif mode in ("dynamic", "high-dynamic-range"):
        scale = np.array([1.0, 1e-2, 1e-4, 1e-6], np.float32)[(k & np.uint64(3)).astype(np.int64)]
        re = np.where(k & np.uint64(1), -scale, scale).astype(np.float32) * np.ones((batch, 1), np.float32)
        im = np.where(k & np.uint64(2), np.float32(0.5) * scale, np.float32(-0.5) * scale).astype(np.float32) \
            * np.ones((batch, 1), np.float32)
    elif mode == "near-cancellation":
        odd = (k & np.uint64(1)).astype(bool) & np.ones((batch, 1), bool)
        re = np.where(odd, np.float32(-1.0) + np.float32(1e-6), np.float32(1.0)).astype(np.float32)
        im = np.where(odd, np.float32(0.5) - np.float32(1e-6), np.float32(-0.5)).astype(np.float32)
    elif mode == "ofdm":
        x = app_hash(b, k)
        q = np.array([-3.0, -1.0, 1.0, 3.0], np.float32)
        kk = k.astype(np.int64) * np.ones((batch, 1), np.int64)
        guard = (kk == 0) | (kk < n // 16) | (kk >= n - n // 16)
        pilot = (kk % 12) == 0
        qr = q[(x & 3).astype(np.int64)] * np.float32(0.31622776)
        qi = q[((x >> 2) & 3).astype(np.int64)] * np.float32(0.31622776)
        pr = np.where(x & 1, 1.0, -1.0).astype(np.float32)
        pi_ = np.where(x & 2, 1.0, -1.0).astype(np.float32)
        re = np.where(guard, 0.0, np.where(pilot, pr, qr)).astype(np.float32)
        im = np.where(guard, 0.0, np.where(pilot, pi_, qi)).astype(np.float32)
    elif mode == "radar":
        x = app_hash(b, k)
        fr = [1.0 / 16, 1.0 / 5, 1.0 / 3, 0.62]
        am = [1.0, 0.5, 0.25, 0.125]
        dop = [0.0, 1.0 / 64, -1.0 / 128, 3.0 / 256]
        frf = np.float32(fr)
        domf = np.float32(dop)
        sr = np.zeros((batch, n))
        si = np.zeros((batch, n))
        for t in range(4):
            ph = 2.0 * np.pi * (float(frf[t]) * k.astype(np.float64) + float(domf[t]) * b.astype(np.float64)) \
                + (t * 0.7 + ((x >> 8) & 255).astype(np.float64) / 255.0 * 0.3)
            sr += am[t] * np.cos(ph)
            si += am[t] * np.sin(ph)
        re = (np.float32(0.25) * sr.astype(np.float32)).astype(np.float32)
        im = (np.float32(0.25) * si.astype(np.float32)).astype(np.float32)
    elif mode == "dl":
        xb = app_hash(b, k // np.uint64(8))
        mag = ((xb >> 8) & 255).astype(np.float32) / np.float32(255.0)
        phs = ((xb >> 16) & 3).astype(np.int64)
        c = np.array([1.0, 0.0, -1.0, 0.0], np.float32)
        s = np.array([0.0, 1.0, 0.0, -1.0], np.float32)
        re = mag * c[phs]
        im = mag * s[phs]
    elif mode == "zero":
        pass
    else:
        raise ValueError(mode)
    out = np.empty((batch, 2 * n), np.float32)
    out[:, 0::2] = re
    out[:, 1::2] = im
    return out


# ------------------------------------------------------------------ seeded benchmark inputs


def cfg1_input(n: int = 1024, batch: int = 256, seed: int = 0) -> np.ndarray:
    """Plain C2C: Re/Im i.i.d. U[-1, 1), interleaved [batch][2n]."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, size=(batch, 2 * n)).astype(np.float32)


def grid_seed(n: int, batch: int) -> int:
    """Per-point seed of the 49-point grid: 1000*log2(n) + log2(batch) + 1."""
    return 1000 * int(round(math.log2(n))) + int(round(math.log2(batch))) + 1


def normal_input(n: int, batch: int, seed: int) -> np.ndarray:
    """Re/Im i.i.d. N(0, 1), interleaved float32 [batch][2n]."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal(size=(batch, 2 * n)).astype(np.float32)


def real_input(n: int, batch: int, seed: int) -> np.ndarray:
    """Real rows U[-1, 1), float32 [batch][n]."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, size=(batch, n)).astype(np.float32)


def half_spectrum_input(n: int, batch: int, seed: int) -> np.ndarray:
    """Hermitian half spectrum [batch][n+2] = rfft of seeded reals, DC/Nyquist imag zeroed."""
    X = np.fft.rfft(real_input(n, batch, seed).astype(np.float64), axis=-1)
    X[:, 0] = X[:, 0].real
    X[:, -1] = X[:, -1].real
    return to_interleaved(X)


GRID_N = [64, 128, 256, 512, 1024, 2048, 4096]
GRID_B = [1, 4, 16, 64, 256, 1024, 4096]


def ragged_requests(count: int = 256, seed: int = 7):
    """Ragged mix: log2 n ~ U{6..12}, batch = round(2^U(0,9)), plus OFDM-like 2048 x 1400,
    radar-like 512 x 4096 and spectral-layer-like 1024 x 6144 groups."""
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(count - 3):
        n = 1 << int(rng.integers(6, 13))
        b = max(1, int(round(2.0 ** rng.uniform(0.0, 9.0))))
        reqs.append((n, b))
    reqs += [(2048, 14 * 100), (512, 4096), (1024, 8 * 768)]
    return reqs


def long_batch(n: int) -> int:
    """batch with batch * n = 2^26 complex values."""
    return (1 << 26) // n
