# -*- coding: utf-8 -*-
"""Pin the float64 oracle (oracle/ssq_oracle.py) against ssqueezepy's own
float64 outputs stored in tests/golden/ (generated by make_golden.py)."""
import os

import numpy as np
import pytest

from oracle import ssq_oracle as O
from ssqueezepy_b200 import _params as P
from tests._cases import WAVS, CWT_CASES, STFT_CASES, oracle_kind, rel_l2, chirp_signal


def _cwt_case(g, name):
    wk, st, sqf, mr, pad, flip = [str(v) for v in g[f'{name}/cfg']]
    x = g[f'{name}/x']
    scales = g[f'{name}/scales']
    ssq_freqs = g[f'{name}/ssq_freqs'][::-1]  # ascending, as squeezed
    _, scaletype, _, nv = P.process_scales(scales, len(x), get_params=True)
    const = P.squeeze_weights(scales, scaletype, nv, 'cwt')
    sqtype = scaletype if sqf == 'None' else sqf
    return dict(x=x, kind=oracle_kind(wk), scales=scales, ssq_freqs=ssq_freqs,
                const=const, pad=pad, flip=(flip == 'True'),
                logscale=sqtype.startswith('log'), scaletype=scaletype, nv=nv,
                wk=wk)


@pytest.mark.parametrize('name', CWT_CASES)
def test_oracle_ssq_cwt_matches_reference(golden_transforms, name):
    g = golden_transforms
    c = _cwt_case(g, name)
    Tx, Wx, w = O.ssq_cwt(c['x'], *c['kind'], c['scales'], c['ssq_freqs'],
                          c['const'], padtype=c['pad'], logscale=c['logscale'],
                          flipud=c['flip'])
    assert rel_l2(Wx, g[f'{name}/Wx']) < 1e-13
    assert rel_l2(Tx, g[f'{name}/Tx']) < 1e-12
    if f'{name}/w' in g:
        wr = g[f'{name}/w']
        fin = np.isfinite(wr)
        assert np.array_equal(fin, np.isfinite(w))
        assert np.allclose(w[fin], wr[fin], rtol=1e-9, atol=0)


@pytest.mark.parametrize('name', CWT_CASES)
def test_oracle_icwt_matches_reference(golden_transforms, name):
    g = golden_transforms
    c = _cwt_case(g, name)
    wav = P.Wavelet((WAVS[c['wk']][0], dict(WAVS[c['wk']][1], dtype='float64')))
    Cpsi = P.adm_ssq(wav)
    x = O.icwt(g[f'{name}/Wx'], c['scales'], c['scaletype'], c['nv'], Cpsi,
               x_mean=c['x'].mean())
    assert np.allclose(x, g[f'{name}/icwt'], rtol=1e-12, atol=1e-12)


def test_oracle_batched_matches_reference(golden_transforms):
    g = golden_transforms
    x, scales = g['b0/x'], g['b0/scales']
    _, st, _, nv = P.process_scales(scales, x.shape[-1], get_params=True)
    const = P.squeeze_weights(scales, st, nv, 'cwt')
    Tx, Wx, _ = O.ssq_cwt(x, 'morlet', (6.,), scales, g['b0/ssq_freqs'][::-1],
                          const)
    assert rel_l2(Wx, g['b0/Wx']) < 1e-13
    assert rel_l2(Tx, g['b0/Tx']) < 1e-12


@pytest.mark.parametrize('name', STFT_CASES)
def test_oracle_ssq_stft_matches_reference(golden_transforms, name):
    g = golden_transforms
    win, n_fft, win_len, hop = [str(v) for v in g[f'{name}/cfg']]
    n_fft, win_len, hop = int(n_fft), int(win_len), int(hop)
    window, dwin = P.get_window(None if win == 'None' else win, win_len,
                                n_fft, derivative=True)
    Tx, Sx, w, Sfs = O.ssq_stft(g[f'{name}/x'], window, dwin, n_fft, hop)
    assert rel_l2(Sx, g[f'{name}/Sx']) < 1e-13
    assert rel_l2(Tx, g[f'{name}/Tx']) < 1e-12
    assert np.allclose(Sfs, g[f'{name}/Sfs'])
    if f'{name}/w' in g:
        wr = g[f'{name}/w']
        fin = np.isfinite(wr)
        assert np.array_equal(fin, np.isfinite(w))
        assert np.allclose(w[fin], wr[fin], rtol=1e-9, atol=1e-12)


def test_oracle_full_size_digest_10k(golden_digests):
    """N=10,000 chirp, Morlet mu=6, log-piecewise scales, log ssq_freqs."""
    d = golden_digests
    x = chirp_signal(10000, seed=0)
    scales = d['d10k/scales']
    _, st, _, nv = P.process_scales(scales, 10000, get_params=True)
    const = P.squeeze_weights(scales, st, nv, 'cwt')
    Tx, Wx, w = O.ssq_cwt(x, 'morlet', (6.,), scales, d['d10k/ssq_freqs'][::-1],
                          const)
    assert np.allclose(np.linalg.norm(Wx, axis=1), d['d10k/Wx_rownorm'],
                       rtol=1e-11)
    assert np.allclose(Wx.sum(1), d['d10k/Wx_rowsum'], rtol=1e-9, atol=1e-9)
    assert np.allclose(np.linalg.norm(Tx, axis=1), d['d10k/Tx_rownorm'],
                       rtol=1e-9, atol=1e-12)
    assert np.allclose(Tx.sum(1), d['d10k/Tx_rowsum'], rtol=1e-9, atol=1e-9)
    r = int(d['d10k/Tx_row_idx'])
    assert np.allclose(Tx[r][::16], d['d10k/Tx_row'], rtol=1e-9, atol=1e-12)
    fin = np.isfinite(w)
    assert fin.sum() == int(d['d10k/w_finite'])


@pytest.mark.parametrize('padtype', ['reflect', 'zero', 'symmetric', 'wrap'])
@pytest.mark.parametrize('N', [300, 1000])
def test_cwt_adjoint_is_the_transpose(padtype, N):
    """Re <g, cwt(x)> == <x, cwt_adjoint(g)> (the dot-product test), float64."""
    rng = np.random.default_rng(N)
    scales = np.geomspace(1.5, N / 8, 40)
    x = rng.standard_normal((2, N))
    g = rng.standard_normal((2, 40, N)) + 1j * rng.standard_normal((2, 40, N))
    Wx, _ = O.cwt(x, 'morlet', (6.,), scales, padtype=padtype, derivative=False)
    gx = O.cwt_adjoint(g, 'morlet', (6.,), scales, padtype=padtype)
    lhs = np.real(np.vdot(g, Wx))
    rhs = float(np.sum(x * gx))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_squeeze_and_icwt_adjoints_are_transposes():
    rng = np.random.default_rng(5)
    na, N = 30, 200
    W = rng.standard_normal((na, N)) + 1j * rng.standard_normal((na, N))
    k = rng.integers(0, na, (na, N))
    use = rng.random((na, N)) > 0.2
    c = rng.random(na)
    gT = rng.standard_normal((na, N)) + 1j * rng.standard_normal((na, N))
    T = O.squeeze(W, k, use, c)
    gW = O.squeeze_adjoint(gT, k, use, c)
    assert abs(np.real(np.vdot(gT, T)) - np.real(np.vdot(gW, W))) < 1e-10 * np.abs(T).sum()
    w = rng.random(na)
    gx = rng.standard_normal(N)
    xr = (w[:, None] * W.real).sum(0)
    gW2 = O.icwt_adjoint(gx, w)
    assert abs(float(gx @ xr) - np.real(np.vdot(gW2, W))) < 1e-10 * np.abs(xr).sum()


@pytest.mark.parametrize('padtype', ['reflect', 'zero'])
@pytest.mark.parametrize('hop', [1, 3])
def test_stft_adjoint_is_the_transpose(padtype, hop):
    from scipy.signal import get_window
    rng = np.random.default_rng(hop)
    N, n_fft = 500, 64
    win = get_window('hann', n_fft, fftbins=True)
    x = rng.standard_normal(N)
    Sx, _ = O.stft(x, win, win, n_fft, hop=hop, padtype=padtype)
    g = rng.standard_normal(Sx.shape) + 1j * rng.standard_normal(Sx.shape)
    gx = O.stft_adjoint(g, win, n_fft, N, hop=hop, padtype=padtype)
    lhs = np.real(np.vdot(g, Sx))
    assert abs(lhs - float(x @ gx)) <= 1e-10 * np.abs(g).sum() * np.abs(Sx).max()


def _issq_inputs():
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        'make_golden', os.path.join(os.path.dirname(__file__), 'golden', 'make_golden.py'))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.issq_inputs()


def test_oracle_issq_matches_golden():
    g = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'issq.npz'))
    Tc, Ts, cc, cw = _issq_inputs()
    for key, wav in (('gmw', ('gmw', {})), ('morlet6', ('morlet', {'mu': 6.}))):
        scale = 2 / P.adm_ssq(P.Wavelet(wav))
        assert rel_l2(O.issq(Tc, scale), g['cwt_full_' + key]) < 1e-12
        assert rel_l2(O.issq(Tc, scale, cc, cw), g['cwt_comp_' + key]) < 1e-12
    win, _ = P.get_window('hann', 256, n_fft=256)
    scale = 2 / win[128]
    assert rel_l2(O.issq(Ts, scale), g['stft_full_hann256']) < 1e-12
    assert rel_l2(O.issq(Ts, scale, cc, cw), g['stft_comp_hann256']) < 1e-12


def test_oracle_ridges_match_golden():
    g = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'ridges.npz'))
    for dt in ('f64', 'f32'):
        T = g['Tf'] if dt == 'f64' else g['Tf'].astype(np.complex64)
        for ax, tr in (('log', 'cwt'), ('lin', 'stft')):
            for nr, bw in ((1, 15), (2, 4)):
                key = '%s_%s_r%d' % (dt, ax, nr)
                i, f, e = O.extract_ridges(T, g['scales_' + ax], 2., nr, bw, tr)
                assert np.array_equal(i, g[key + '_idx']), key
                assert np.array_equal(f, g[key + '_f']), key
                assert np.allclose(e, g[key + '_e'], rtol=1e-6 if dt == 'f32' else 1e-14), key


def test_bin_parity_counts_and_edges():
    """The bin-parity checker: the oracle's own bins give no mismatch; a
    moved bin counts as `other`; an entry whose w sits at its rounding edge,
    given the bin across the edge, counts as `near_edge`."""
    from ssqueezepy_b200 import _transforms as T
    from tests._cases import chirp_signal
    N = 2000
    x = chirp_signal(N).astype(np.float32).astype(np.float64)
    wav = P.Wavelet(('morlet', {'mu': 6.}))
    s = P.process_scales('log-piecewise', N, wav, nv=32).ravel()
    fp = T._ssq_plan(wav, 'log-piecewise', N, 32, None, 'peak', 'reflect', 1.)
    W, dW = O.cwt(x, 'morlet', (6.,), s)
    g = 10 * P.EPS32
    w = O.phase_cwt(W, dW, g)
    use = np.abs(W) > g
    k = np.where(use, O.bin_index(np.where(use, w, 1.), fp['f_asc'], True, True), 0xFFFF)
    r = O.bin_parity(k, W, dW, fp['f_asc'], True, True, g)
    assert r['mismatched'] == 0 and r['mask_mismatched'] == 0
    i, j = np.argwhere(use)[100]
    k2 = k.copy()
    k2[i, j] = (k2[i, j] + 3) % len(s)
    r = O.bin_parity(k2, W, dW, fp['f_asc'], True, True, g)
    assert r['mismatched'] == 1 and r['other'] == 1
    # every entry's edge lies within half a bin of it
    e = O.bin_edge_w(w[use], fp['f_asc'], True)
    ratio = np.log2(e / w[use]) / np.log2(fp['f_asc'][1] / fp['f_asc'][0])
    assert np.all(np.abs(ratio) <= 0.5 + 1e-9)
    ei = O.bin_edge_w(np.array([w[i, j]]), fp['f_asc'], True)[0]
    dW2 = dW.copy()
    dW2[i, j] *= ei / w[i, j]
    w2 = O.phase_cwt(W, dW2, g)[i, j]
    kk = O.bin_index(np.array([w2]), fp['f_asc'], True, True)[0]
    res = []
    for d in (-1, 1):
        k3 = k.copy()
        k3[i, j] = kk + d
        res.append(O.bin_parity(k3, W, dW2, fp['f_asc'], True, True, g))
    assert any(r['near_edge'] == 1 and r['other'] == 0 for r in res), res


def test_cpu_path_port_tracks_float64_oracle():
    """The timed CPU arm (the reference's float32 CPU execution): Wx at the
    float32 level of the float64 oracle, Tx at the reference's own float32
    level (bin flips of entries near an edge, ~1e-3)."""
    from oracle.ssq_cpu_path import SsqCwtCpu
    from ssqueezepy_b200 import _transforms as T
    from tests._cases import chirp_signal, rel_l2
    N = 3000
    x = chirp_signal(N).astype(np.float32)
    wav = P.Wavelet(('gmw', {'gamma': 3., 'beta': 60.}))
    s = P.process_scales('log-piecewise', N, wav, nv=32).ravel()
    fp = T._ssq_plan(wav, 'log-piecewise', N, 32, None, 'peak', 'reflect', 1.)
    port = SsqCwtCpu(N, 'gmw_l1', (3., 60.), s, fp['mode'], fp['bp'], fp['const'])
    Tx, Wx = port(x)
    To, Wo, _ = O.ssq_cwt(x.astype(np.float64), 'gmw_l1', (3., 60.), s, fp['f_asc'],
                          fp['const'], gamma=10 * O.EPS32)
    assert rel_l2(Wx, Wo) < 1e-5
    assert rel_l2(Tx, To) < 1e-2
    Tx2, _ = port(x)
    assert np.array_equal(Tx, Tx2)  # deterministic: columns are independent
