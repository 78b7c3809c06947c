"""Seeded synthetic workloads of the benchmark configurations (no datasets:
every input is generated from a fixed seed with the stated shape and value
distribution)."""
from __future__ import annotations

import math

import numpy as np


def _is_smooth13(n: int) -> bool:
    for p in (2, 3, 5, 7, 11, 13):
        while n % p == 0:
            n //= p
    return n == 1


def _is_prime(n: int) -> bool:
    if n < 2:
        return False
    if n % 2 == 0:
        return n == 2
    d = 3
    while d * d <= n:
        if n % d == 0:
            return False
        d += 2
    return True


def _nearest(n: int, pred, lo: int, hi: int) -> int:
    for d in range(0, hi):
        for c in (n - d, n + d):
            if lo <= c <= hi and pred(c):
                return c
    raise ValueError("no candidate")


def mixed_lengths(count: int = 20000, seed: int = 5, lo: int = 16, hi: int = 65536):
    """Line lengths log-uniform in [lo, hi]; by a seeded draw 70% snapped to
    the nearest 13-smooth length, 15% to the nearest prime and 15% to the
    nearest composite with a prime factor above 13."""
    rng = np.random.default_rng(seed)
    raw = np.exp(rng.uniform(math.log(lo), math.log(hi), count))
    cls = rng.uniform(0.0, 1.0, count)
    out = []
    for r, c in zip(raw, cls):
        n = int(round(r))
        if c < 0.70:
            out.append(_nearest(n, _is_smooth13, lo, hi))
        elif c < 0.85:
            out.append(_nearest(n, _is_prime, lo, hi))
        else:
            out.append(_nearest(n, lambda m: m > 3 and not _is_prime(m) and not _is_smooth13(m),
                                lo, hi))
    return np.asarray(out, dtype=np.int64)


def packed_offsets(lengths) -> np.ndarray:
    """Lines stored back to back: offset of each line in complex elements."""
    lengths = np.asarray(lengths, dtype=np.int64)
    off = np.zeros(len(lengths), dtype=np.int64)
    if len(lengths) > 1:
        off[1:] = np.cumsum(lengths[:-1])
    return off


def normal_complex(n: int, seed: int) -> np.ndarray:
    """iid N(0,1) real and imaginary parts as complex64."""
    rng = np.random.default_rng(seed)
    x = np.empty(n, dtype=np.complex64)
    x.real = rng.standard_normal(n, dtype=np.float32)
    x.imag = rng.standard_normal(n, dtype=np.float32)
    return x


def uniform_complex(n: int, seed: int) -> np.ndarray:
    """iid uniform[-1, 1) real and imaginary parts as complex64."""
    rng = np.random.default_rng(seed)
    x = np.empty(n, dtype=np.complex64)
    x.real = rng.uniform(-1.0, 1.0, n).astype(np.float32)
    x.imag = rng.uniform(-1.0, 1.0, n).astype(np.float32)
    return x


def hdr_complex(n: int, seed: int) -> np.ndarray:
    """High-dynamic-range input: magnitudes log-uniform in [1e-6, 1e6],
    phases uniform in [0, 2 pi), as complex128 (round to the storage
    precision before use)."""
    rng = np.random.default_rng(seed)
    mag = np.exp(rng.uniform(math.log(1e-6), math.log(1e6), n))
    ph = rng.uniform(0.0, 2.0 * math.pi, n)
    return mag * np.exp(1j * ph)


def fft_flops(n: int) -> float:
    """The 5 N log2 N convention for one complex transform of length N."""
    return 5.0 * n * math.log2(n) if n > 1 else 0.0


def serving_requests(count: int, seed: int = 9, max_bytes: int = 64 << 20):
    """Requests of the serving configuration: C2C or R2C, forward or inverse;
    1D length log-uniform in [64, 2^22], 2D sides from {64, ..., 4096} or 3D
    cubes from {32, 64, 128, 256}; batch uniform in 1..64; precision 80% f32,
    10% f64, 10% df64 (df64 is C2C only, like the reference).  The batch is
    reduced until one request holds at most max_bytes of input."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        r = rng.uniform()
        if r < 1 / 3:
            shape = [int(round(math.exp(rng.uniform(math.log(64), math.log(1 << 22)))))]
        elif r < 2 / 3:
            shape = [int(rng.choice([64, 128, 256, 512, 1024, 2048, 4096])) for _ in range(2)]
        else:
            c = int(rng.choice([32, 64, 128, 256]))
            shape = [c, c, c]
        batch = int(rng.integers(1, 65))
        u = rng.uniform()
        prec = 0 if u < 0.8 else (1 if u < 0.9 else 2)
        real = rng.uniform() < 0.5 and prec != 2
        inverse = rng.uniform() < 0.5
        kind = (2 if inverse else 1) if real else 0
        bpc = 8 if prec == 0 else 16
        while batch > 1 and int(np.prod(shape)) * batch * bpc > max_bytes:
            batch //= 2
        out.append({"kind": kind, "shape": shape, "batch": batch, "precision": prec,
                    "inverse": inverse})
    return out
