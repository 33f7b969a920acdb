# -*- coding: utf-8 -*-
"""Inverse STFT (`istft`, _stft.py:184-256; `ssqb_istft`). CPU: the oracle
against the reference's outputs (tests/golden/istft.npz, made by
tests/golden/make_golden.py), argument checks. GPU: every fixture case,
batches, and the stft -> istft round trip at the full N=160,000 size."""
import ctypes
import os

import numpy as np
import pytest

from ssqueezepy_b200 import _lib as L
from ssqueezepy_b200 import _params as P
from tests._cases import rel_l2, chirp_signal
from tests.golden.make_golden import ISTFT_CASES

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'istft.npz')


def _case_args(case):
    name, N, n_fft, win_len, hop, win, Ni, mod, wexp, dt = case
    return name, dict(window=win, n_fft=n_fft, win_len=win_len, hop_len=hop, N=Ni,
                      modulated=mod, win_exp=wexp)


@pytest.mark.parametrize('case', ISTFT_CASES, ids=[c[0] for c in ISTFT_CASES])
def test_oracle_matches_reference(case):
    from oracle import ssq_oracle as O
    g = np.load(GOLD)
    name, kw = _case_args(case)
    win, _ = P.get_window(kw['window'], kw['win_len'], kw['n_fft'])
    x = O.istft(g[name + '/Sx'], win, kw['n_fft'], kw['hop_len'], kw['N'],
                kw['modulated'], kw['win_exp'])
    assert x.shape == g[name + '/x'].shape
    assert rel_l2(x, g[name + '/x']) <= 1e-15


def test_istft_argument_checks():
    import ssqueezepy_b200 as sb
    S = np.zeros((33, 10), np.complex128)
    with pytest.raises(ValueError):
        sb.istft(S.real)
    with pytest.raises(NotImplementedError):
        sb.istft(S, n_fft=2000)         # not a power of two, above 1024
    with pytest.raises(NotImplementedError):
        sb.istft(S, n_fft=128)          # rows != n_fft//2 + 1
    with pytest.raises(ValueError):
        sb.istft(S, hop_len=4, N=30)    # 9 * 4 > 29: frames past the signal


def test_istft_abi_rejects_bad_arguments():
    lib = L.load()
    p = ctypes.c_void_p(8)

    def call(**kw):
        a = dict(S=p, B=1, n_fft=64, nf=10, hop=1, N=10, mod=1, wa=p, w1=p, tiny=1e-300,
                 prec=L.F64, x=p, ws=p, wsb=1 << 30)
        a.update(kw)
        return lib.ssqb_istft(a['S'], a['B'], a['n_fft'], a['nf'], a['hop'], a['N'],
                              a['mod'], a['wa'], a['w1'], a['tiny'], a['prec'], a['x'],
                              a['ws'], a['wsb'], None)
    assert call(S=None) == L.EINVAL
    assert call(B=0) == L.EINVAL
    assert call(n_fft=2000) == L.EUNSUPPORTED      # not a power of two, above 1024
    assert call(n_fft=3) == L.EUNSUPPORTED
    assert call(n_fft=8192) == L.EUNSUPPORTED
    assert call(nf=11) == L.EINVAL                # (11 - 1) * 1 > 9
    assert call(tiny=-1.) == L.EINVAL
    assert call(prec=7) == L.EINVAL
    assert call(wsb=16) == L.EWORKSPACE
    assert lib.ssqb_istft_workspace_bytes(2, 64, 10, L.F64) == 2 * 64 * 10 * 8
    assert lib.ssqb_istft_workspace_bytes(2, 64, 10, L.F32) == 2 * 64 * 10 * 4


#### GPU ######################################################################
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize('case', ISTFT_CASES, ids=[c[0] for c in ISTFT_CASES])
def test_istft_matches_reference(case):
    _gpu()
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    name, kw = _case_args(case)
    x = sb.istft(g[name + '/Sx'], **kw)
    ref = g[name + '/x']
    assert isinstance(x, np.ndarray) and x.dtype == ref.dtype and x.shape == ref.shape
    # float64: sums in another order; float32: the reference sums in float32
    assert rel_l2(x, ref) <= (1e-13 if ref.dtype == np.float64 else 2e-6)


@pytest.mark.gpu
def test_istft_batch_equals_single_and_keeps_tensors():
    torch = _gpu()
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    S = np.stack([g['a/Sx'], 2 * g['a/Sx'], g['a/Sx'].conj()])
    St = torch.as_tensor(S, device='cuda')
    xb = sb.istft(St, n_fft=64, N=300)
    assert xb.is_cuda and tuple(xb.shape) == (3, 300)
    for i in range(3):
        xi = sb.istft(S[i], n_fft=64, N=300)
        assert np.array_equal(xb[i].cpu().numpy(), xi)


@pytest.mark.gpu
@pytest.mark.parametrize('dtype, tol', [('float64', 1e-12), ('float32', 1e-5)])
def test_stft_istft_round_trip_full_size(dtype, tol):
    """istft(stft(x)) = x at the STFT workload's size (N=160,000, hann,
    n_fft=512, hop 1), and with hop 64."""
    _gpu()
    import ssqueezepy_b200 as sb
    x = chirp_signal(160000, seed=2).astype(dtype)
    for hop in (1, 64):
        Sx = sb.stft(x, 'hann', n_fft=512, hop_len=hop, dtype=dtype)
        xr = sb.istft(Sx, 'hann', n_fft=512, hop_len=hop, N=len(x)).cpu().numpy()
        assert rel_l2(xr, x) <= tol, hop
