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


def test_higher_order_needs_a_gmw():
    import ssqueezepy_b200 as sb
    x = np.zeros(64)
    with pytest.raises(ValueError):
        sb.cwt(x, 'morlet', order=1)
    with pytest.raises(ValueError):
        sb.ssq_cwt(x, 'morlet', order=(0, 1))


def test_struct_carries_the_coefficients():
    from ssqueezepy_b200 import _lib as L
    w = P.Wavelet(('gmw', {'order': (0, 1, 2)}))
    cw = L.wavelet_struct(w)
    assert cw.npoly == 3 and np.allclose(list(cw.kc)[:3], w.poly())
    assert list(cw.kc)[3:] == [0.] * 5
    assert L.wavelet_struct(P.Wavelet('gmw')).npoly == 0
    assert L.wavelet_struct(P.Wavelet('morlet')).npoly == 0


#### GPU ######################################################################
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


W64 = ('gmw', {'dtype': 'float64'})


@pytest.mark.gpu
def test_cwt_order2_matches_reference():
    _gpu()
    import ssqueezepy_b200 as sb
    g = golden('higher')
    Wx, sc = sb.cwt(g['x'], W64, order=2, astensor=False)
    assert sc.shape == (g['scales'].shape[0], 1)
    assert np.allclose(sc, g['scales'], rtol=1e-12, atol=0)
    assert rel_l2(Wx, g['cwt_o2_Wx']) <= 1e-10


@pytest.mark.gpu
def test_cwt_average_of_orders_matches_reference():
    _gpu()
    import ssqueezepy_b200 as sb
    g = golden('higher')
    Wx, _ = sb.cwt(g['x'], W64, order=(0, 1, 2), astensor=False)
    assert rel_l2(Wx, g['cwt_avg012_Wx']) <= 1e-10
    Wx, _ = sb.cwt(g['x'], W64, order=range(3), average=True, astensor=False)
    assert rel_l2(Wx, g['cwt_avg012_Wx']) <= 1e-10


@pytest.mark.gpu
def test_ssq_cwt_average_of_orders_matches_reference():
    _gpu()
    import ssqueezepy_b200 as sb
    g = golden('higher')
    Tx, Wx, f, sc = sb.ssq_cwt(g['x'], W64, order=(0, 1), astensor=False)
    assert np.allclose(f, g['ssq_avg01_f'], rtol=1e-12, atol=0)
    assert rel_l2(Tx, g['ssq_avg01_Tx']) <= 1e-9


@pytest.mark.gpu
def test_cwt_orders_unaveraged_are_the_single_orders():
    _gpu()
    import ssqueezepy_b200 as sb
    g = golden('higher')
    Ws, sc = sb.cwt(g['x'], W64, order=(1, 2), average=False, astensor=False)
    assert isinstance(Ws, list) and len(Ws) == 2
    assert rel_l2(Ws[1], g['cwt_o2_Wx']) <= 1e-10
    W1, _ = sb.cwt(g['x'], ('gmw', {'dtype': 'float64', 'order': 1}),
                   scales=sc, astensor=False)
    assert rel_l2(Ws[0], W1) <= 1e-14


@pytest.mark.gpu
def test_cwt_order2_float32_within_the_float32_bar():
    _gpu()
    import ssqueezepy_b200 as sb
    g = golden('higher')
    Wx, _ = sb.cwt(g['x'].astype(np.float32), 'gmw', order=2, astensor=False)
    assert Wx.dtype == np.complex64
    assert rel_l2(Wx, g['cwt_o2_Wx']) <= 1e-5


@pytest.mark.gpu
def test_cwt_higher_order_gradient_is_the_adjoint():
    """The loss Re<G, Wx> is linear in x, so its gradient g satisfies
    <g, x> = loss(x) for every x: the adjoint transform carries the
    polynomial too."""
    torch = _gpu()
    import ssqueezepy_b200 as sb
    rng = np.random.default_rng(5)
    x = torch.tensor(rng.standard_normal(512), device='cuda', requires_grad=True)
    Wx, _ = sb.cwt(x, W64, order=(0, 2))
    G = torch.tensor(rng.standard_normal(tuple(Wx.shape)) +
                     1j * rng.standard_normal(tuple(Wx.shape)), device='cuda')
    loss = (G.conj() * Wx).real.sum()
    loss.backward()
    lin = float((x.grad * x.detach()).sum())
    assert abs(lin - float(loss)) <= 1e-10 * abs(float(loss))


def test_oracle_restates_the_reference():
    """The oracle's order-k GMW (generalized Laguerre polynomial from scipy)
    and its mean over orders against the reference's transforms."""
    from oracle import ssq_oracle as O
    g = golden('higher')
    sc = g['scales'].ravel()
    # scipy's Laguerre recurrence and the reference's power sum round
    # differently where the polynomial's terms cancel: 1e-10 of the peak
    assert np.abs(O.psih('gmw_l1', (3., 60., 1), g['psih_w']) - g['psih_o1']).max() \
        <= 1e-10 * np.abs(g['psih_o1']).max()
    assert np.abs(O.psih('gmw_l2', (3., 60., 3), g['psih_w']) - g['psih_o3e']).max() \
        <= 1e-10 * np.abs(g['psih_o3e']).max()
    Wx, _ = O.cwt(g['x'], 'gmw_l1', (3., 60., 2), sc, derivative=False)
    assert rel_l2(Wx, g['cwt_o2_Wx']) <= 1e-12
    Wx, _ = O.cwt_higher_order(g['x'], 'gmw_l1', (3., 60.), (0, 1, 2), sc,
                               derivative=False)
    assert rel_l2(Wx, g['cwt_avg012_Wx']) <= 1e-12


def test_host_polynomial_equals_the_oracle_laguerre():
    """Wavelet.poly (used by the kernels) against scipy's generalized
    Laguerre polynomial in the oracle, orders 1..7, both norms. The power sum
    in 2 w^gamma cancels more with each order (its terms grow far above
    their sum near the peak), so the two evaluations part by about
    8x per order: 4e-14 of the peak at k = 1, 3e-9 at k = 7."""
    from oracle import ssq_oracle as O
    ws = np.linspace(0, 8, 401)
    for norm, kind in (('bandpass', 'gmw_l1'), ('energy', 'gmw_l2')):
        for k in range(1, P.MAX_GMW_ORDER + 1):
            w = P.Wavelet(('gmw', {'order': k, 'norm': norm, 'dtype': 'float64'}))
            ref = O.psih(kind, (3., 60., k), ws)
            tol = 2e-14 * 8.**k
            assert np.abs(w.fn(ws) - ref).max() <= tol * np.abs(ref).max(), (norm, k)
