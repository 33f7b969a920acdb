# -*- coding: utf-8 -*-
"""The reference's CPU execution of ssq_cwt, restated for timing: float32
data, `SSQ_PARALLEL=1`, `cache_wavelet=True` (the configuration of the
reference's own benchmark, examples/benchmarks.py:30-37).

TEST INFRASTRUCTURE ONLY: bench.py's reference arm and CPU baseline time it;
the product (`ssqueezepy_b200`) never imports it and has no CPU fallback.

It does the work the reference does, in the same order and precision:
reflect padding (utils/common.py:54-158), a float32 FFT of the padded
signal, the cached float32 wavelet bank times the spectrum and its inverse
FFT along rows, the same product times i xi and a second inverse FFT
(_cwt.py:167-177), both through scipy.fft (pocketfft, the reference's CPU
FFT) over every host thread; then the column-parallel squeeze of
algos.py:879-895 / 913-924 (numba prange there, OpenMP C here,
oracle/ssq_cpu.c). Host parameters come in as arguments, as the cache
holds them in the reference after the warm-up calls.
"""
import ctypes
import os
import subprocess

import numpy as np
from scipy import fft as sfft

from oracle import ssq_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'ssq_cpu.c')
LIB = os.path.join(HERE, '_lib', 'libssqcpu.so')


def build(force=False):
    """Compile the OpenMP squeeze (gcc) into oracle/_lib/."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    tmp = LIB + '.tmp'
    subprocess.run(['gcc', '-O3', '-fopenmp', '-shared', '-fPIC', SRC, '-o', tmp, '-lm'],
                   check=True, capture_output=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        f = _lib.ssq_cpu_squeeze
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        f.argtypes = [P, P, P, P, I, I, ctypes.c_longlong, D, I, D, D, D, D, I, I, I]
        f.restype = None
    return _lib


class SsqCwtCpu:
    """One float32 ssq_cwt of length N with a cached wavelet bank.

    kind, params: the oracle's wavelet (`psih`); scales (na,); bin mode and
    parameters as `ssqueezepy_b200._params.bin_params` gives them; const
    (na,) per-row weights; flipud as ssq_cwt's default."""

    def __init__(self, N, kind, params, scales, mode, bp, const, flipud=True,
                 workers=None):
        self.N = N
        self.Npad, self.n1, self.n2 = O.p2up(N)
        Ps, xi = O.psih_bank(kind, params, scales, self.Npad)
        self.Psih = Ps.astype(np.float32)                 # the cached bank
        self.ixi = (1j * xi).astype(np.complex64)
        self.na = len(scales)
        self.const = np.asarray(const, np.float32)
        self.mode, self.bp, self.flipud = mode, bp, flipud
        self.workers = workers or os.cpu_count() or 1
        self.gamma = 10 * O.EPS32
        # work buffers reused across calls (fresh 600 MB arrays per call would
        # time page faults, not the transform)
        self.B1 = np.empty((self.na, self.Npad), np.complex64)
        self.B2 = np.empty_like(self.B1)
        _load()

    def __call__(self, x):
        x = np.asarray(x, np.float32)
        xp = np.pad(x, (self.n1, self.n2), mode='reflect')
        xh = sfft.fft(xp, workers=self.workers)
        np.multiply(self.Psih, xh, out=self.B1)
        np.multiply(self.B1, self.ixi, out=self.B2)
        W = sfft.ifft(self.B1, axis=-1, workers=self.workers, overwrite_x=True)
        dW = sfft.ifft(self.B2, axis=-1, workers=self.workers, overwrite_x=True)
        Wx = W[:, self.n1:self.n1 + self.N]
        dWx = dW[:, self.n1:self.n1 + self.N]
        assert W.dtype == np.complex64 and W.strides == dW.strides
        Tx = np.zeros((self.na, self.N), np.complex64)
        if self.mode == 1:
            v0, v1, d0, d1, idx1 = self.bp
        else:
            v0, d0 = self.bp[0], self.bp[1]
            v1 = d1 = 0.
            idx1 = 0
        _lib.ssq_cpu_squeeze(Wx.ctypes.data, dWx.ctypes.data, Tx.ctypes.data,
                             self.const.ctypes.data, self.na, self.N,
                             W.strides[0] // W.itemsize, self.gamma,
                             int(self.mode), float(v0), float(v1), float(d0), float(d1),
                             int(idx1), self.na - 1, 1 if self.flipud else 0)
        return Tx, Wx
