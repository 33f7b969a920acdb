# -*- coding: utf-8 -*-
"""Shared definitions of the golden cases (see tests/golden/make_golden.py)."""
import numpy as np

WAVS = {
    'morlet6': ('morlet', {'mu': 6.}),
    'morlet13.4': ('morlet', {'mu': 13.4}),
    'morlet5': ('morlet', {'mu': 5.}),
    'gmw3_60': ('gmw', {'gamma': 3., 'beta': 60.}),
    'gmw3_8': ('gmw', {'gamma': 3., 'beta': 8.}),
}

CWT_CASES = ['c0', 'c1', 'c2', 'c3', 'c4']
STFT_CASES = ['s0', 's1', 's2', 's3']


def oracle_kind(key):
    name, opts = WAVS[key]
    if name == 'morlet':
        return 'morlet', (opts['mu'],)
    return 'gmw_l1', (opts['gamma'], opts['beta'])


def chirp_signal(N, seed=0):
    """Linear chirp 0.01->0.2 cycles/sample + AM tone at 0.3 + N(0, 0.1^2)
    noise (float64), seeded."""
    t = np.arange(N, dtype=np.float64)
    rng = np.random.default_rng(seed)
    return (np.cos(2 * np.pi * (0.01 * t + 0.19 * t**2 / (2 * N)))
            + (0.5 + 0.5 * np.cos(2 * np.pi * 0.001 * t))
            * np.cos(2 * np.pi * 0.3 * t)
            + 0.1 * rng.standard_normal(N))


def rel_l2(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
