# -*- coding: utf-8 -*-
"""Higher-order generalized Morse wavelets (`order=k`, `order=(k0, k1, ...)`).

An order-k GMW is the order-0 exponential times a Laguerre polynomial in
2 w^gamma (_gmw.py:268-347); averaging the transforms over several orders
(cwt_higher_order, _cwt.py:517-610) is averaging the wavelets, since the CWT
is linear in the wavelet. CPU: the wavelet samples and constants against
fixtures from the reference. GPU: cwt / ssq_cwt against the reference's
float64 transforms of the same signal."""
import os

import numpy as np
import pytest

from ssqueezepy_b200 import _params as P
from tests._cases import rel_l2

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'higher.npz')


def golden(name):
    return np.load(GOLD)


def test_order1_wavelet_matches_reference():
    g = golden('higher')
    w = P.Wavelet(('gmw', {'order': 1, 'dtype': 'float64'}))
    got = w.fn(g['psih_w'])
    assert np.abs(got - g['psih_o1']).max() <= 1e-13 * np.abs(g['psih_o1']).max()


def test_order3_energy_wavelet_matches_reference():
    g = golden('higher')
    w = P.Wavelet(('gmw', {'order': 3, 'norm': 'energy', 'dtype': 'float64'}))
    got = w.fn(g['psih_w'])
    assert np.abs(got - g['psih_o3e']).max() <= 1e-12 * np.abs(g['psih_o3e']).max()


def test_order0_constants_are_the_base_norm():
    """k = 0: L = [1], so kc = [2] (bandpass peak 2) and the order-0 energy
    norm sqrt(2 pi gamma 2^r / Gamma(r))."""
    from scipy.special import gamma as G
    assert np.allclose(P.gmw_k_constants(3., 60., 0), [2.])
    r = (2 * 60. + 1) / 3.
    assert np.allclose(P.gmw_k_constants(3., 60., 0, 'energy'),
                       [np.sqrt(2 * np.pi * 3. * 2**r / G(r))])


def test_order_tuple_averages_coefficients():
    w = P.Wavelet(('gmw', {'order': (0, 2), 'dtype': 'float64'}))
    k0 = P.gmw_k_constants(3., 60., 0)
    k2 = P.gmw_k_constants(3., 60., 2)
    assert np.allclose(w.poly(), (np.pad(k0, (0, 2)) + k2) / 2)
    # averaged wavelet = mean of the per-order wavelets
    ws = np.linspace(0, 10, 101)
    a = P.Wavelet(('gmw', {'order': 0, 'dtype': 'float64'})).fn(ws)
    b = P.Wavelet(('gmw', {'order': 2, 'dtype': 'float64'})).fn(ws)
    assert np.allclose(w.fn(ws), (a + b) / 2, rtol=1e-12, atol=1e-14)


def test_order_checks():
    assert P._check_order([3]) == 3
    assert P._check_order(range(3)) == (0, 1, 2)
    with pytest.raises(NotImplementedError):
        P._check_order(P.MAX_GMW_ORDER + 1)
    with pytest.raises(NotImplementedError):
        P._check_order((0, -1))
    assert P.Wavelet(('gmw', {'order': 0})).poly() is None


def test_higher_order_band_covers_the_wavelet():
    """The polynomial's zeros and its shifted peak: everything outside the
    band is below the floor relative to the peak."""
    w = P.Wavelet(('gmw', {'order': 3, 'dtype': 'float64'}))
    lo, hi = w.band()
    grid = np.geomspace(1e-6, 1e3, 20000)
    v = np.abs(w.fn(grid))
    out = (grid < lo) | (grid > hi)
    assert v[out].max() <= 1e-12 * v.max() * 10
