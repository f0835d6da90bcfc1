"""Seeded synthetic inputs for benchmarks and tools.

The device generators (``ms_gpu_gen_*``) draw value i from a counter-based
splitmix64 stream, so a column is a function of (seed, i).  Skewed
distributions are drawn by inverse CDF from a threshold table: a draw u maps
to the smallest k with u < table[k]; table[k] = floor(2^64 * F(k)) computed in
80-bit extended precision, the last entry 2^64 - 1.
"""
from __future__ import annotations

import numpy as np

_TWO64 = np.longdouble(18446744073709551616.0)


def _thresholds(cdf: np.ndarray) -> np.ndarray:
    t = cdf * _TWO64
    out = np.empty(len(cdf), np.uint64)
    full = (cdf >= 1) | (t >= np.longdouble(18446744073709551615.0))
    # exact conversion of values below 2^64: split into two 32-bit halves
    tt = np.where(full, np.longdouble(0), np.floor(t))
    hi = np.floor(tt / np.longdouble(4294967296.0))
    lo = tt - hi * np.longdouble(4294967296.0)
    out[:] = (hi.astype(np.uint64) << np.uint64(32)) | lo.astype(np.uint64)
    out[full] = np.uint64(0xFFFFFFFFFFFFFFFF)
    return out


def zipf_table(s: float, n_vals: int) -> np.ndarray:
    """P(k) proportional to (k+1)^-s over k in [0, n_vals)."""
    w = np.power(np.arange(1, n_vals + 1, dtype=np.longdouble), -np.longdouble(s))
    acc = np.cumsum(w)
    t = _thresholds(acc / acc[-1])
    t[-1] = np.uint64(0xFFFFFFFFFFFFFFFF)
    return t


def geom_table(p: float, max_len: int = 4096) -> np.ndarray:
    """P(G = k) = p (1-p)^k, k >= 0, truncated where the CDF reaches 1."""
    q = np.longdouble(1) - np.longdouble(p)
    qk = np.cumprod(np.full(max_len, q, dtype=np.longdouble))
    t = _thresholds(np.longdouble(1) - qk)
    full = np.flatnonzero(t == np.uint64(0xFFFFFFFFFFFFFFFF))
    k = int(full[0]) if len(full) else max_len - 1
    t = t[: k + 1].copy()
    t[-1] = np.uint64(0xFFFFFFFFFFFFFFFF)
    return t
