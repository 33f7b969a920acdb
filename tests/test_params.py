# -*- coding: utf-8 -*-
"""Host float64 parameter layer vs ssqueezepy's own values (golden)."""
import numpy as np
import pytest

from ssqueezepy_b200 import _params as P
from tests._cases import WAVS


def _wav(key):
    name, opts = WAVS[key]
    return P.Wavelet((name, dict(opts, dtype='float64')))


def test_p2up(golden_params):
    for k, v in golden_params.items():
        if k.startswith('p2up/'):
            assert tuple(P.p2up(int(k.split('/')[1]))) == tuple(v)


@pytest.mark.parametrize('key', list(WAVS))
def test_scales_bit_exact(golden_params, key):
    w = _wav(key)
    n = 0
    for k, ref in golden_params.items():
        parts = k.split('/')
        if parts[0] != 'scales' or parts[1] != key:
            continue
        N, st = int(parts[2]), parts[3]
        if ref.size == 0:  # the reference raises for this combination
            with pytest.raises(Exception):
                P.process_scales(st, N, w, nv=32)
            continue
        s = P.process_scales(st, N, w, nv=32).ravel()
        dk = f'scales_digest/{key}/{N}/{st}'
        if dk in golden_params:
            size, s1, s2 = golden_params[dk]
            assert s.size == int(size)
            s = np.hstack([s[:64], s[-64:]])
        assert np.array_equal(s, ref), k
        n += 1
    assert n > 20


@pytest.mark.parametrize('key', list(WAVS))
def test_ssq_freqs_and_bins(golden_params, key):
    """ssq_freqs agree to an ulp or two ('energy' integrates numba-evaluated
    samples; numba's exp and numpy's differ in the last bit), bin parameters
    likewise."""
    w = _wav(key)
    n = 0
    for k, ref in golden_params.items():
        parts = k.split('/')
        if parts[0] != 'ssq_freqs' or parts[1] != key:
            continue
        N, st, sqs, mr = int(parts[2]), parts[3], parts[4], parts[5]
        scales = P.process_scales(st, N, w, nv=32)
        f = P.compute_associated_frequencies(scales, N, w, sqs, mr, True, 1.,
                                             'cwt')
        if f.size > 2048:
            f = np.hstack([f[:64], f[-64:]])
        if mr != 'energy':
            assert np.array_equal(f, ref), k
        else:
            assert np.allclose(f, ref, rtol=1e-14, atol=1e-16), k
        bk = 'binp/' + k[10:]
        if bk in golden_params and f.size <= 2048:
            mode, p = P.bin_params(f, True)
            p = np.array([float(v) for v in p])[:len(golden_params[bk])]
            assert np.allclose(p, golden_params[bk], rtol=1e-13, atol=1e-15), bk
        n += 1
    assert n > 10


@pytest.mark.parametrize('key', list(WAVS))
def test_adm_ssq(golden_params, key):
    assert np.isclose(P.adm_ssq(_wav(key)), float(golden_params[f'adm_ssq/{key}']),
                      rtol=1e-13)


def test_dtype_defaults():
    w = P.Wavelet()
    assert w.dtype == 'float32' and w.name == 'GMW L1'
    assert P.Wavelet(('gmw', {'norm': 'energy'})).dtype == 'float64'
    assert P.Wavelet('morlet').config['mu'] == 13.4


def test_bad_args():
    with pytest.raises(ValueError):
        P.Wavelet('bump_nope')
    with pytest.raises(ValueError):
        P.process_scales('logg', 100, P.Wavelet())
    with pytest.raises(ValueError):
        P.Wavelet(('gmw', {'gamma': -1}))
    with pytest.raises(Exception):
        P.process_fs_and_t(None, np.array([0, 1, 3.]), 3)


def test_ssq_plan_weights_follow_scale_array():
    """log-piecewise scales: the squeeze weight is ln2/nv per row, nv read
    from the scale array (32 below the transition, 8 above), as ssqueeze
    re-derives it (ssqueezing.py:168-169, 124-128)."""
    from ssqueezepy_b200 import _transforms as T
    w = P.Wavelet(('morlet', {'mu': 6.}))
    fp = T._ssq_plan(w, 'log-piecewise', 10000, 32, 'log', 'peak', 'reflect', 1.)
    c = fp['const']
    s = P.process_scales('log-piecewise', 10000, w, nv=32).ravel()
    idx = P.logscale_transition_idx(s)
    assert idx is not None
    assert np.allclose(c[:idx], np.log(2) / 32) and np.allclose(c[idx:], np.log(2) / 8)


def test_float32_scale_arrays_plan_like_float64():
    """Scales handed back at float32 (as ssq_cwt returns them for float32
    data) keep their log-piecewise type: the transition is found at float32
    tolerances, as the reference does (cwt_utils.py:375-394), for the squeeze
    bins and weights and for icwt's pieces."""
    import numpy as np
    from ssqueezepy_b200 import _params as P
    from ssqueezepy_b200 import _transforms as T
    w = P.Wavelet('gmw', N=1024)
    sc64 = P.process_scales('log-piecewise', 1024, w, nv=32).ravel()
    out = []
    for sc in (sc64, sc64.astype(np.float32)):
        sp = T._scales_plan(sc, 1024, w, None)
        fp = T._ssq_plan(w, sc, 1024, None, None, 'peak', 'reflect', 1.0, sp)
        ip = T._icwt_plan(w, sc, 1024, None, True)
        out.append((sp['scaletype'], fp['mode'], fp['bp'][4], len(ip['weights']),
                    ip['mean_mult']))
    assert out[0] == out[1] == ('log-piecewise', 1, out[0][2], len(sc64), 2.0)
