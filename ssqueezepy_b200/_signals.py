# -*- coding: utf-8 -*-
"""Seeded synthetic signals of the benchmark workloads (the reference ships
comparable generators in ssqueezepy/_test_signals.py: linear chirps
:226-264, hyperbolic chirps :266-282). No public dataset is involved.

* `chirp_tone(N, seed)`: linear chirp 0.01 -> 0.2 cycles/sample over the
  whole length, plus a 0.3 cycles/sample tone with 0.5 + 0.5 cos(2 pi 0.001 t)
  amplitude modulation, plus N(0, 0.1^2) noise.
* `chirp_mix(N, rng)`: 1-3 components, each a linear or hyperbolic chirp with
  start / end frequencies uniform in [0.005, 0.45] cycles/sample and
  amplitude uniform in [0.2, 1], plus white noise at an SNR uniform in
  [0, 20] dB.
* `uneven_batch(n, lo, hi, seed)`: n signals of `chirp_mix` with lengths
  uniform in [lo, hi].
All are generated in float64; callers cast.
"""
import numpy as np

__all__ = ['chirp_tone', 'chirp_mix', 'uneven_batch', 'same_length_batch']


def chirp_tone(N, seed=0):
    t = np.arange(N, dtype=np.float64)
    rng = np.random.default_rng(seed)
    return (np.cos(2 * np.pi * (0.01 * t + 0.19 * t**2 / (2 * N)))
            + (0.5 + 0.5 * np.cos(2 * np.pi * 0.001 * t))
            * np.cos(2 * np.pi * 0.3 * t)
            + 0.1 * rng.standard_normal(N))


def _phase_linear(t, N, f0, f1):
    # f(t) = f0 + (f1 - f0) t / N
    return 2 * np.pi * (f0 * t + (f1 - f0) * t**2 / (2 * N))


def _phase_hyperbolic(t, N, f0, f1):
    # f(t) = A / (B - t)^2 through f(0) = f0 and f(N) = f1; its phase is
    # 2 pi A (1/(B - t) - 1/B)
    r = np.sqrt(f0 / f1)
    if abs(1 - r) < 1e-9:
        return 2 * np.pi * f0 * t
    B = N / (1 - r)
    A = f0 * B * B
    return 2 * np.pi * A * (1 / (B - t) - 1 / B)


def chirp_mix(N, rng):
    t = np.arange(N, dtype=np.float64)
    x = np.zeros(N)
    for _ in range(int(rng.integers(1, 4))):
        f0, f1 = rng.uniform(0.005, 0.45, 2)
        amp = rng.uniform(0.2, 1.0)
        ph = (_phase_linear if rng.random() < 0.5 else _phase_hyperbolic)(t, N, f0, f1)
        x += amp * np.cos(ph)
    snr_db = rng.uniform(0, 20)
    sigma = np.sqrt(np.var(x) / 10**(snr_db / 10))
    return x + sigma * rng.standard_normal(N)


def uneven_batch(n=256, lo=4096, hi=65536, seed=1234):
    rng = np.random.default_rng(seed)
    lengths = rng.integers(lo, hi + 1, n)
    return [chirp_mix(int(N), rng) for N in lengths]


def same_length_batch(n, N, seed):
    rng = np.random.default_rng(seed)
    return np.stack([chirp_mix(N, rng) for _ in range(n)])
