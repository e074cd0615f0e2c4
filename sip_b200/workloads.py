"""Seeded synthetic workloads of the FFT path (no dataset exists for it).

* ``uneven_batch_set`` — the uneven batch: 1D C2C complex64 transforms whose
  lengths are drawn log-uniformly from [64, 65536] and snapped to the nearest
  2^a 3^b 5^c 7^d, each drawn length getting a Zipf(1.2) batch count capped at
  512, until the batch counts sum to the requested total (20 000).
* ``chirp_noise`` — complex chirp plus white noise at a given SNR (serving).
"""
from __future__ import annotations

import math

import numpy as np


def smooth_numbers(lo: int, hi: int, primes=(2, 3, 5, 7)) -> list[int]:
    out = {1}
    for p in primes:
        cur = list(out)
        for v in cur:
            x = v * p
            while x <= hi:
                out.add(x)
                x *= p
    return sorted(v for v in out if lo <= v <= hi)


def uneven_batch_set(total: int = 20000, lo: int = 64, hi: int = 65536, zipf_a: float = 1.2, cap: int = 512,
                     seed: int = 2024) -> list[tuple[int, int]]:
    """[(length, batch), ...] sorted by length; batches sum to `total`."""
    rng = np.random.default_rng(seed)
    smooth = np.array(smooth_numbers(lo, hi), dtype=np.float64)
    logs = np.log(smooth)
    groups: dict[int, int] = {}
    acc = 0
    while acc < total:
        u = rng.uniform(math.log(lo), math.log(hi))
        n = int(smooth[int(np.argmin(np.abs(logs - u)))])
        b = int(min(rng.zipf(zipf_a), cap, total - acc))
        groups[n] = groups.get(n, 0) + b
        acc += b
    return sorted(groups.items())


def uneven_flops_bytes(groups) -> tuple[float, int]:
    fl = sum(5.0 * n * math.log2(n) * b for n, b in groups)
    by = sum(16 * n * b for n, b in groups)
    return fl, by


def chirp_noise(n: int, rows: int, snr_db: float, seed: int) -> np.ndarray:
    """Complex linear chirp (random start/stop frequency) plus complex white noise."""
    rng = np.random.default_rng(seed)
    t = np.arange(n) / n
    f0 = rng.uniform(0, 0.25 * n, size=(rows, 1))
    f1 = rng.uniform(0.25 * n, 0.5 * n, size=(rows, 1))
    phase = 2 * np.pi * (f0 * t + 0.5 * (f1 - f0) * t * t)
    s = np.exp(1j * phase)
    p_noise = 10 ** (-snr_db / 10.0)
    noise = np.sqrt(p_noise / 2) * (rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n)))
    return (s + noise).astype(np.complex64)
