# -*- coding: utf-8 -*-
"""Phase transforms by differences along time: `ssq_cwt(difftype='phase' |
'numeric', get_w=True)`, `phase_cwt(difftype='phase')`, `phase_cwt_num`
(_ssq_cwt.py:420-586; `ssqb_phase_diff`). CPU: the oracle against the
reference's outputs (tests/golden/difftype.npz, made by
tests/golden/make_golden.py), argument checks. GPU: the same fixtures."""
import ctypes
import os
import warnings

import numpy as np
import pytest

from ssqueezepy_b200 import _lib as L
from tests._cases import rel_l2

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'difftype.npz')
W64 = ('gmw', {'dtype': 'float64'})
GAMMA64 = 10 * np.finfo(np.float64).eps


def _close_w(a, b, tol):
    """Equal inf masks (|Wx| < gamma) and finite values within `tol`."""
    a, b = np.asarray(a), np.asarray(b)
    assert np.array_equal(np.isinf(a), np.isinf(b))
    f = np.isfinite(b)
    return rel_l2(a[f], b[f]) <= tol


def test_oracle_phase_transforms_match_reference():
    from oracle import ssq_oracle as O
    g = np.load(GOLD)
    W0 = g['cwt/Wx']
    assert _close_w(O.phase_unwrap(W0, np.sqrt(np.finfo(np.float64).eps)),
                    g['phase_cwt/w'], 1e-14)
    assert _close_w(O.phase_numeric(W0, 1., 4, GAMMA64), g['phase_cwt_num/w'], 1e-14)


def test_difftype_argument_checks():
    from ssqueezepy_b200 import _transforms as T
    import ssqueezepy_b200 as sb
    with pytest.raises(ValueError):
        sb.ssq_cwt(np.zeros(64), difftype='phase')            # needs get_w
    with pytest.raises(ValueError):
        sb.ssq_cwt(np.zeros(64), difftype='numeric', difforder=3, get_w=True)
    with pytest.raises(ValueError):
        sb.ssq_cwt(np.zeros(64), difftype='other', get_w=True)
    assert T._check_ssq_args('sum', 'peak', 'numeric', True, None) == 4
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter('always')
        T._check_ssq_args('sum', 'peak', 'trig', True, 2)
    assert any('ignored' in str(r.message) for r in rec)
    with pytest.raises(ValueError):
        sb.phase_cwt(np.zeros((2, 8), np.complex128), None, difftype='numeric')
    with pytest.raises(ValueError):
        sb.phase_cwt_num(np.zeros((2, 8), np.complex128), 1., difforder=3)


def test_phase_diff_abi_rejects_bad_arguments():
    lib = L.load()
    p = ctypes.c_void_p(8)

    def call(**kw):
        a = dict(W=p, B=1, na=4, ncol=64, col0=0, M=64, mode=1, order=4, dt=1., gamma=1e-6,
                 prec=L.F64, w=p)
        a.update(kw)
        return lib.ssqb_phase_diff(a['W'], a['B'], a['na'], a['ncol'], a['col0'], a['M'],
                                   a['mode'], a['order'], a['dt'], a['gamma'], a['prec'],
                                   a['w'], None)
    assert call(W=None) == L.EINVAL
    assert call(M=1) == L.EINVAL
    assert call(col0=4) == L.EINVAL            # 4 + 64 > 64
    assert call(col0=-1, M=8) == L.EINVAL
    assert call(mode=3) == L.EINVAL
    assert call(mode=2, order=3) == L.EINVAL
    assert call(mode=2, dt=0.) == L.EINVAL
    assert call(prec=9) == L.EINVAL


#### GPU ######################################################################
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


@pytest.mark.gpu
def test_ssq_cwt_difftype_phase_matches_reference():
    _gpu()
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    Tx, Wx, f, sc, w = sb.ssq_cwt(g['x'], W64, nv=8, difftype='phase', get_w=True,
                                  astensor=False)
    assert np.allclose(f, g['phase/f'], rtol=1e-12, atol=0)
    assert _close_w(w, g['phase/w'], 1e-12)
    assert rel_l2(Tx, g['phase/Tx']) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize('order', [1, 2, 4])
def test_ssq_cwt_difftype_numeric_matches_reference(order):
    _gpu()
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    k = 'num%d/' % order
    Tx, Wx, f, sc, w = sb.ssq_cwt(g['x'], W64, nv=8, difftype='numeric', difforder=order,
                                  get_w=True, astensor=False)
    assert np.allclose(f, g[k + 'f'], rtol=1e-12, atol=0)
    assert _close_w(w, g[k + 'w'], 1e-12)
    assert rel_l2(Tx, g[k + 'Tx']) <= 1e-9
    assert Wx.shape == tuple(g['num4/Wx_shape'])
    assert rel_l2(Wx[0], g['num4/Wx_row0']) <= 1e-12


@pytest.mark.gpu
def test_phase_cwt_phase_and_numeric_match_reference():
    _gpu()
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    W0 = g['cwt/Wx']
    w = sb.phase_cwt(W0, None, difftype='phase').cpu().numpy()
    assert _close_w(w, g['phase_cwt/w'], 1e-13)
    w = sb.phase_cwt_num(W0, 1., difforder=4).cpu().numpy()
    assert _close_w(w, g['phase_cwt_num/w'], 1e-13)


@pytest.mark.gpu
def test_phase_diff_float32_against_the_oracle():
    """float32 Wx, float64 arithmetic: within float32 rounding of the oracle
    on the same (rounded) input."""
    _gpu()
    import ssqueezepy_b200 as sb
    from oracle import ssq_oracle as O
    g = np.load(GOLD)
    W32 = g['cwt/Wx'].astype(np.complex64)
    gam = np.sqrt(np.finfo(np.float32).eps)
    w = sb.phase_cwt(W32, None, difftype='phase').cpu().numpy()
    assert w.dtype == np.float32
    assert _close_w(w, O.phase_unwrap(W32.astype(np.complex128), gam), 1e-6)
    w = sb.phase_cwt_num(W32, 1., difforder=2).cpu().numpy()
    ref = O.phase_numeric(W32.astype(np.complex128), 1., 2, 10 * np.finfo(np.float32).eps)
    assert _close_w(w, ref, 1e-6)
