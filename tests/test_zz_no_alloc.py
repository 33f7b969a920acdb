# -*- coding: utf-8 -*-
"""ssqb_cwt_noalloc: the CWT entry point for callers that cannot allocate
device memory on their call path (a plugin whose host application owns all
device memory, or a streaming loop that cannot take cudaMalloc's implicit
synchronization). It keeps its scratch in a fixed 16 MiB module array
instead of a caller workspace; results must equal ssqb_cwt's.

The array keeps the previous call's contents, so each comparison runs after
a larger call on a different signal has left them stale. Free device memory
must not change across the first call in the process.

This file is collected last so that a failure here, in a run that stops at
the first failure, comes after every other test has run."""
import ctypes

import numpy as np
import pytest
import torch

from ssqueezepy_b200 import _lib as L
from ssqueezepy_b200 import _params as P
from tests._cases import chirp_signal, rel_l2

pytestmark = pytest.mark.gpu

PRECS = {'F32X': (L.F32X, np.float32, torch.complex64),
         'F32': (L.F32, np.float32, torch.complex64),
         'F64': (L.F64, np.float64, torch.complex128)}


def _setup(N, prec, seed):
    code, xdt, cdt = PRECS[prec]
    w = P.Wavelet(('gmw', {'gamma': 3., 'beta': 60., 'dtype': 'float64'}))
    sc, st, na, nv = P.process_scales('log-piecewise', N, w, nv=32, get_params=True)
    f = P.compute_associated_frequencies(sc, N, w, st, 'peak', True, 1., 'cwt')
    mode, bp = P.bin_params(f, True)
    Npad, n1, _ = P.p2up(N)
    dev = torch.device('cuda', 0)
    x = torch.as_tensor(chirp_signal(N, seed=seed).astype(xdt), device=dev)
    gamma = 10 * (P.EPS64 if prec == 'F64' else P.EPS32)
    ip = L.idx_pitch(N)
    wsb = L.load().ssqb_cwt_workspace_bytes(1, N, Npad, na, code)
    return dict(N=N, na=na, Npad=Npad, n1=n1, x=x, dev=dev, code=code, gamma=gamma, ip=ip,
                sc=torch.as_tensor(sc.ravel(), dtype=torch.float64, device=dev),
                cw=L.wavelet_struct(w), cb=L.make_bins(mode, bp, na, True),
                Wx=torch.empty((1, na, N), dtype=cdt, device=dev),
                idx=torch.empty((1, na, ip), dtype=torch.uint16, device=dev),
                ws=torch.empty(wsb, dtype=torch.uint8, device=dev), wsb=wsb)


def _call(c, noalloc):
    lib = L.load()
    c['Wx'].fill_(float('nan'))
    c['idx'].fill_(0x7777)
    args = (L.ptr(c['x']), 1, c['N'], c['Npad'], c['n1'], 1, 0, L.ptr(c['sc']), c['na'],
            c['cw'], 1.0, c['cb'], c['gamma'], c['code'], L.ptr(c['Wx']), None, None,
            L.ptr(c['idx']), c['ip'])
    if noalloc:
        rc = lib.ssqb_cwt_noalloc(*args, L.stream_ptr())
    else:
        rc = lib.ssqb_cwt(*args, L.ptr(c['ws']), c['wsb'], L.stream_ptr())
    L.check(rc, 'cwt')
    torch.cuda.synchronize()
    return c['Wx'].cpu().numpy(), c['idx'].cpu().numpy()[..., :c['N']]


@pytest.fixture(scope='module')
def cuda():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    torch.cuda.set_device(0)
    return L.load()


@pytest.mark.parametrize('prec', list(PRECS))
def test_noalloc_equals_cwt_on_two_calls_in_a_row(cuda, prec):
    """A N=160,000 call (padded 262,144: two-pass, most of the scratch) on
    one signal, then two N=10,000 calls on another: each equals ssqb_cwt on
    the same input, and the first noalloc call leaves free device memory
    unchanged (outputs, inputs and ssqb_cwt's workspace are allocated and its
    kernels loaded before the measurement)."""
    big, small = _setup(160000, prec, 3), _setup(10000, prec, 4)
    ref_big, ref_small = _call(big, noalloc=False), _call(small, noalloc=False)
    free0 = torch.cuda.mem_get_info()[0]
    W, k = _call(big, noalloc=True)
    assert torch.cuda.mem_get_info()[0] == free0
    assert np.isfinite(W).all() and rel_l2(W, ref_big[0]) <= 1e-5
    assert np.array_equal(k, ref_big[1])
    for _ in range(2):
        W, k = _call(small, noalloc=True)
        assert np.isfinite(W).all()
        assert rel_l2(W, ref_small[0]) <= 1e-5  # the float32 Wx bar of the other tests
        assert np.array_equal(k, ref_small[1])
    assert L.device_status() == 0


def test_noalloc_rejects_calls_beyond_its_scratch(cuda):
    lib = L.load()
    assert lib.ssqb_cwt_noalloc_max_bytes() == 16 << 20
    c = _setup(160000, 'F32X', 3)
    B = 4  # needs 4 x 262144 x 48 bytes
    rc = lib.ssqb_cwt_noalloc(L.ptr(c['x']), B, c['N'], c['Npad'], c['n1'], 1, 0,
                              L.ptr(c['sc']), c['na'], c['cw'], 1.0, c['cb'],
                              10 * P.EPS32, L.F32X, ctypes.c_void_p(8), None, None,
                              None, 0, L.stream_ptr())
    assert rc == L.EINVAL
    assert b'scratch' in lib.ssqb_last_error()


def test_noalloc_reports_its_own_argument_errors(cuda):
    """Bad sizes are reported as ssqb_cwt reports them, not as a missing
    workspace."""
    lib = L.load()
    c = _setup(10000, 'F32X', 3)

    def call(B=1, Npad=c['Npad'], prec=L.F32X):
        return lib.ssqb_cwt_noalloc(L.ptr(c['x']), B, c['N'], Npad, c['n1'], 1, 0,
                                    L.ptr(c['sc']), c['na'], c['cw'], 1.0, c['cb'],
                                    10 * P.EPS32, prec, L.ptr(c['Wx']), None, None,
                                    L.ptr(c['idx']), c['ip'], L.stream_ptr())
    assert call(Npad=12000) == L.EUNSUPPORTED
    assert b'power of two' in lib.ssqb_last_error()
    assert call(B=0) == L.EINVAL
    assert b'>= 1' in lib.ssqb_last_error()
    assert call(prec=7) == L.EINVAL
    assert b'precision' in lib.ssqb_last_error()
