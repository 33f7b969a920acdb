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
