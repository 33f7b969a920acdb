# -*- coding: utf-8 -*-
"""ssqb_cwt_noalloc: the CWT entry point for callers that cannot allocate
device memory on their call path (a plugin whose host application owns all
device memory, or a streaming loop that cannot take cudaMalloc's implicit
synchronization). It keeps its scratch in a fixed 16 MiB module array
instead of a caller workspace; results must equal ssqb_cwt's.

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


def _setup(N, dtype='float32'):
    w = P.Wavelet(('gmw', {'gamma': 3., 'beta': 60., 'dtype': dtype}))
    sc, st, na, nv = P.process_scales('log-piecewise', N, w, nv=32, get_params=True)
    f = P.compute_associated_frequencies(sc, N, w, st, 'peak', True, 1., 'cwt')
    mode, bp = P.bin_params(f, True)
    Npad, n1, _ = P.p2up(N)
    dev = torch.device('cuda', 0)
    x = torch.as_tensor(chirp_signal(N, seed=3).astype(np.float32), device=dev)
    return dict(N=N, na=na, Npad=Npad, n1=n1, x=x, dev=dev,
                sc=torch.as_tensor(sc.ravel(), dtype=torch.float64, device=dev),
                cw=L.wavelet_struct(w), cb=L.make_bins(mode, bp, na, True))


def _outputs(c):
    ip = L.idx_pitch(c['N'])
    Wx = torch.full((1, c['na'], c['N']), float('nan'), dtype=torch.complex64,
                    device=c['dev'])
    idx = torch.full((1, c['na'], ip), 0x7777, dtype=torch.uint16, device=c['dev'])
    return Wx, idx, ip


def _call(c, noalloc):
    lib = L.load()
    Wx, idx, ip = _outputs(c)
    args = (L.ptr(c['x']), 1, c['N'], c['Npad'], c['n1'], 1, 0, L.ptr(c['sc']), c['na'],
            c['cw'], 1.0, c['cb'], 10 * P.EPS32, L.F32X, L.ptr(Wx), None, None,
            L.ptr(idx), ip)
    if noalloc:
        rc = lib.ssqb_cwt_noalloc(*args, L.stream_ptr())
    else:
        wsb = lib.ssqb_cwt_workspace_bytes(1, c['N'], c['Npad'], c['na'], L.F32X)
        ws = torch.empty(wsb, dtype=torch.uint8, device=c['dev'])
        rc = lib.ssqb_cwt(*args, L.ptr(ws), wsb, L.stream_ptr())
    L.check(rc, 'cwt')
    torch.cuda.synchronize()
    return Wx.cpu().numpy(), idx.cpu().numpy()[..., :c['N']]


@pytest.fixture(scope='module')
def cuda():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    torch.cuda.set_device(0)
    return L.load()


@pytest.mark.parametrize('N', [10000, 160000])
def test_noalloc_equals_cwt_on_two_calls_in_a_row(cuda, N):
    """N=10,000 (padded 16,384) and N=160,000 (padded 262,144, one row per
    two-pass tile in the fixed scratch): two consecutive calls both give
    ssqb_cwt's Wx and bins."""
    c = _setup(N)
    W_ref, k_ref = _call(c, noalloc=False)
    for _ in range(2):
        W, k = _call(c, noalloc=True)
        assert np.isfinite(W).all()
        assert rel_l2(W, W_ref) <= 1e-5  # the float32 Wx bar of the other tests
        assert np.array_equal(k, k_ref)
    assert L.device_status() == 0


def test_noalloc_rejects_calls_beyond_its_scratch(cuda):
    lib = L.load()
    assert lib.ssqb_cwt_noalloc_max_bytes() == 16 << 20
    c = _setup(160000)
    B = 4  # needs 4 x (4 + 8) MiB
    rc = lib.ssqb_cwt_noalloc(L.ptr(c['x']), B, c['N'], c['Npad'], c['n1'], 1, 0,
                              L.ptr(c['sc']), c['na'], c['cw'], 1.0, c['cb'],
                              10 * P.EPS32, L.F32X, ctypes.c_void_p(8), None, None,
                              None, 0, L.stream_ptr())
    assert rc == L.EINVAL
    assert b'scratch' in lib.ssqb_last_error()
