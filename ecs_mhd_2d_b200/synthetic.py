"""Seeded synthetic initial conditions for the benchmark workloads.

IC(seed, n): numpy default_rng(seed) (PCG64); for each channel and each
half-spectrum mode with 1 <= |k| <= 8 the coefficient is |k|^-2 (a + i b),
a, b ~ N(0, 1); real projection irfft2(rfft2(.)), 2/3 mask (which also removes
the mean), then both channels scaled so that max|omega| = 10 (the reference's
plotting range, jax_scripts/animation.py:36-37).
"""

from __future__ import annotations

import numpy as np


def initial_condition(seed: int, n: int, kmin=1.0, kmax=8.0, amp=10.0):
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n, d=1 / n)
    kx = k.reshape(-1, 1)
    ky = np.abs(k[: n // 2 + 1]).reshape(1, -1)
    kk = np.sqrt(kx * kx + ky * ky)
    band = (kk >= kmin) & (kk <= kmax)
    fields = np.zeros((2, n, n))
    for c in range(2):
        a = rng.standard_normal((n, n // 2 + 1))
        b = rng.standard_normal((n, n // 2 + 1))
        coef = np.where(band, (a + 1j * b) / np.where(band, kk, 1.0) ** 2, 0.0)
        fields[c] = np.fft.irfft2(coef, s=(n, n))
    fields = np.fft.irfft2(np.fft.rfft2(fields), s=(n, n))
    mask = (np.abs(kx) < n / 3) & (ky < n / 3)
    mask[0, 0] = False
    fields = np.fft.irfft2(mask * np.fft.rfft2(fields), s=(n, n))
    fields *= amp / np.max(np.abs(fields[0]))
    return fields


def unit_tangents(seed: int, n: int, count: int):
    """`count` seeded unit-norm flat tangents of length 2 n^2 + 2 ([T, fields, sx] order)."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((count, 2 * n * n + 2))
    return v / np.linalg.norm(v, axis=1, keepdims=True)
