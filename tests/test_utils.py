# -*- coding: utf-8 -*-
"""Host helpers of the path with the reference's interface: `padsignal`
(utils/common.py:54-158) and `get_window` (_stft.py:259-310), against the
reference's outputs (tests/golden/utils.npz, made by
tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import ssqueezepy_b200 as sb
from tests.golden.make_golden import PAD_CASES, WINDOW_CASES

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'utils.npz')


@pytest.mark.parametrize('pt, pl', PAD_CASES)
def test_padsignal_matches_reference(pt, pl):
    g = np.load(GOLD)
    xp, n_up, n1, n2 = sb.padsignal(g['x'], pt, pl, get_params=True)
    assert np.array_equal(xp, g['pad_%s_%s' % (pt, pl)])
    assert [n_up, n1, n2] == list(g['pad_%s_%s_geom' % (pt, pl)])
    assert np.array_equal(sb.padsignal(g['x'][1], pt, pl), g['pad_%s_%s' % (pt, pl)][1])


def test_padsignal_tensor_modes_and_errors():
    import torch
    x = torch.arange(10.)
    assert torch.equal(sb.padsignal(x, 'zero', 16), torch.nn.functional.pad(x, (3, 3)))
    with pytest.raises(ValueError):
        sb.padsignal(x, 'wrap')
    with pytest.raises(ValueError):
        sb.padsignal(np.zeros((2, 2, 2)))


@pytest.mark.parametrize('win, wl, nf', WINDOW_CASES)
def test_get_window_matches_reference(win, wl, nf):
    g = np.load(GOLD)
    w, dw = sb.get_window(win, wl, nf, derivative=True)
    k = '%s_%d_%s' % (win, wl, nf)
    assert np.array_equal(w, g['win_' + k])
    assert np.allclose(dw, g['dwin_' + k], rtol=1e-12, atol=1e-15)
    assert sb.get_window(win, wl, nf, dtype='float32').dtype == np.float32


def test_trigdiff_argument_checks():
    A = np.zeros((2, 64), np.complex128)
    with pytest.raises(NotImplementedError):
        sb.trigdiff(A, transform='stft')
    with pytest.raises(ValueError):
        sb.trigdiff(A, rpadded=True)          # needs N
    with pytest.raises(ValueError):
        sb.trigdiff(np.zeros((2, 2, 64), np.complex128))  # padding takes 1D / 2D
    with pytest.raises(AssertionError):
        sb.trigdiff(np.zeros(64, np.complex128))


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')


@pytest.mark.gpu
def test_trigdiff_matches_reference():
    _gpu()
    from tests._cases import rel_l2
    g = np.load(GOLD)
    A, Ap = g['td_A'], g['td_Ap']
    cases = [(sb.trigdiff(A, fs=2.), 'td_reflect'),
             (sb.trigdiff(A, fs=1., padtype='zero', N=300), 'td_zero_N'),
             (sb.trigdiff(Ap[0], fs=3., rpadded=True, N=300), 'td_rpadded'),
             (sb.trigdiff(Ap, rpadded=True, N=256, n1=100), 'td_rpadded3')]
    for got, key in cases:
        assert got.shape == g[key].shape, key
        assert rel_l2(got, g[key]) <= 1e-12, key
    got32 = sb.trigdiff(A.astype(np.complex64), fs=2.)
    assert got32.dtype == np.complex64 and rel_l2(got32, g['td_reflect']) <= 1e-5


@pytest.mark.gpu
def test_trigdiff_of_padded_cwt_is_its_derivative():
    """What the reference's higher-order ssq_cwt relies on: trigdiff of the
    padded transform equals the transform's frequency-domain derivative
    (the same halved Nyquist bin in both)."""
    _gpu()
    from tests._cases import rel_l2, chirp_signal
    x = chirp_signal(3000, seed=5)
    wav = ('gmw', {'dtype': 'float64'})
    Wp, sc = sb.cwt(x, wav, rpadded=True, astensor=False)
    Wx, _, dWx = sb.cwt(x, wav, derivative=True, astensor=False)
    D = sb.trigdiff(Wp, fs=1., rpadded=True, N=3000)
    assert rel_l2(D, dWx) <= 1e-11
