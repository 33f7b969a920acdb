# -*- coding: utf-8 -*-
"""Batches of uneven-length signals (ssqb_cwt_batch / ssqb_squeeze_batch,
`SsqCwtBatch`). CPU: descriptor layout, argument checks, launch counting,
descriptor packing, the signal family. GPU: each signal's results equal a
one-signal `ssq_cwt` call (the same kernels), and the float64 oracle within
the float32 bars; graph replay repeats the eager results."""
import ctypes

import numpy as np
import pytest

from ssqueezepy_b200 import _lib as L
from ssqueezepy_b200 import _signals as S


def _sig(n=1, N=1000, Npad=2048, na=20, **kw):
    s = np.zeros(n, L.SIG_DTYPE)
    s['N'], s['n1'], s['na'], s['idx_pitch'] = N, (Npad - N) // 2, na, L.idx_pitch(N)
    s['mode'], s['nbins'], s['flipud'] = 0, na, 1
    s['p'] = [[-3., 0.05, 0., 0.]] * n
    s['scales'] = s['weights'] = 8
    for k, v in kw.items():
        s[k] = v
    return s


def _cwt_batch(sigs, Npad=2048, prec=L.F32X, wsb=1 << 30, nsig=None):
    lib = L.load()
    p = ctypes.c_void_p(8)
    return lib.ssqb_cwt_batch(p, sigs.ctypes.data_as(ctypes.c_void_p), p,
                              len(sigs) if nsig is None else nsig, Npad, 1,
                              L.make_wavelet(0, (6., 1e-8, 1., 0.)), 1.0, 1e-6, prec,
                              p, p, p, wsb, None)


def test_descriptor_layout_matches_header():
    assert L.SIG_DTYPE.itemsize == 104
    assert L.SIG_DTYPE.fields['scales'][1] == 24
    assert L.SIG_DTYPE.fields['N'][1] == 40
    assert L.SIG_DTYPE.fields['mode'][1] == 56
    assert L.SIG_DTYPE.fields['p'][1] == 72


@pytest.mark.parametrize('kw, nsig', [
    (dict(), 0),
    (dict(N=3000), None),             # longer than Npad
    (dict(n1=1500), None),            # pad geometry
    (dict(idx_pitch=10), None),
    (dict(na=0), None),
    (dict(nbins=19), None),           # nbins != na
    (dict(mode=5), None),
    (dict(x_off=-1), None),
    (dict(scales=0), None),
])
def test_cwt_batch_rejects_bad_descriptors(kw, nsig):
    assert _cwt_batch(_sig(3, **kw), nsig=nsig) == L.EINVAL
    assert L.load().ssqb_last_error()


def test_cwt_batch_rejects_bad_arguments():
    assert _cwt_batch(_sig(2), prec=L.F64) == L.EUNSUPPORTED
    assert _cwt_batch(_sig(2), Npad=3000) == L.EUNSUPPORTED
    assert _cwt_batch(_sig(2), wsb=64) == L.EWORKSPACE
    lib = L.load()
    p = ctypes.c_void_p(8)
    s = _sig(2)
    assert lib.ssqb_squeeze_batch(p, p, s.ctypes.data_as(ctypes.c_void_p), p, 2, L.F64,
                                  p, None) == L.EUNSUPPORTED
    s['weights'] = 0
    assert lib.ssqb_squeeze_batch(p, p, s.ctypes.data_as(ctypes.c_void_p), p, 2, L.F32,
                                  p, None) == L.EINVAL
    s = _sig(2, na=20000, nbins=20000)
    assert lib.ssqb_squeeze_batch(p, p, s.ctypes.data_as(ctypes.c_void_p), p, 2, L.F32,
                                  p, None) == L.EUNSUPPORTED


def test_batch_workspace_and_launch_count():
    lib = L.load()
    s = _sig(40, N=60000, Npad=1 << 17, na=300)
    ws = lib.ssqb_cwt_batch_workspace_bytes(40, 1 << 17, L.F32X)
    assert ws >= 40 * (1 << 17) * 16 + 2 * (1 << 17) * 16
    n = lib.ssqb_cwt_batch_launches(s.ctypes.data_as(ctypes.c_void_p), 40, 1 << 17,
                                    L.F32X, ws)
    # two x_hat passes per chunk plus two CWT passes per (chunk, row tile)
    assert n >= 2 + 2 * 300 // 16 and n % 2 == 0
    small = _sig(5, N=1000, Npad=2048, na=40)
    assert lib.ssqb_cwt_batch_launches(small.ctypes.data_as(ctypes.c_void_p), 5, 2048,
                                       L.F32X, 1 << 20) == 2  # one pass each
    assert lib.ssqb_cwt_batch_launches(small.ctypes.data_as(ctypes.c_void_p), 5, 2048,
                                       L.F64, 1 << 20) == -1


def test_describe_signals_packs_end_to_end():
    """Descriptors carry each signal's own one-signal ssq_cwt parameters."""
    from ssqueezepy_b200._batch import describe_signals
    from ssqueezepy_b200 import _params as P
    lengths = [5000, 700, 20000, 4100]
    wav = P.Wavelet(('morlet', {'mu': 6.}))
    sig, d = describe_signals(lengths, wav)
    assert list(sig['N']) == lengths
    assert list(sig['x_off']) == [0, 5000, 5700, 25700] and d['n_x'] == sum(lengths)
    na = [P.process_scales('log-piecewise', N, wav, nv=32).size for N in lengths]
    assert list(sig['na']) == na and list(sig['nbins']) == na
    assert list(sig['out_off']) == list(np.cumsum([0] + [a * N for a, N in
                                                           zip(na, lengths)])[:-1])
    pitches = [L.idx_pitch(N) for N in lengths]
    assert list(sig['idx_pitch']) == pitches
    assert list(sig['idx_off']) == list(np.cumsum([0] + [a * p for a, p in
                                                           zip(na, pitches)])[:-1])
    assert list(sig['scales']) == list(np.cumsum([0] + na)[:-1])
    for i, N in enumerate(lengths):
        Npad, n1, _ = P.p2up(N)
        assert sig['n1'][i] == n1 and n1 + N <= Npad
        s64 = P.process_scales('log-piecewise', N, wav, nv=32).ravel()
        assert np.array_equal(d['scales64'][i], s64)
        # log-piecewise bins; N=700 has no transition and gets plain log bins
        assert sig['mode'][i] == (0 if N == 700 else 1) and sig['flipud'][i] == 1
        assert d['ssq_freqs'][i][0] > d['ssq_freqs'][i][-1]   # high to low
        # per-row weights ln2/nv with nv inferred from the scale array
        assert np.allclose(d['weights64'][i][:3], np.log(2) / 32)


def test_uneven_batch_family():
    xs = S.uneven_batch(8, 4096, 65536, seed=1234)
    assert len(xs) == 8 and all(4096 <= len(x) <= 65536 for x in xs)
    assert len(set(len(x) for x in xs)) > 1
    ys = S.uneven_batch(8, 4096, 65536, seed=1234)
    assert all(np.array_equal(a, b) for a, b in zip(xs, ys))
    assert all(np.isfinite(x).all() and x.std() > 0 for x in xs)


#### GPU ######################################################################
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


LENGTHS = [3000, 5000, 4100, 20000, 2900, 11000, 700, 9000]  # Npad 1024..32768


@pytest.mark.gpu
@pytest.mark.parametrize('wavelet', [('morlet', {'mu': 6.}),
                                     ('gmw', {'gamma': 3., 'beta': 60.})])
def test_batch_equals_single_calls(wavelet):
    torch = _gpu()
    import ssqueezepy_b200 as sb
    from ssqueezepy_b200._batch import SsqCwtBatch
    rng = np.random.default_rng(7)
    xs = [S.chirp_mix(N, rng).astype(np.float32) for N in LENGTHS]
    plan = SsqCwtBatch(LENGTHS, wavelet=wavelet)
    outs = plan(xs)
    torch.cuda.synchronize()
    for x, (Tx, Wx, f, sc) in zip(xs, outs):
        T1, W1, f1, s1 = sb.ssq_cwt(x, wavelet=wavelet)
        assert np.array_equal(f, f1)
        assert torch.equal(sc, s1)
        w, w1 = Wx.cpu().numpy(), W1.cpu().numpy()
        t, t1 = Tx.cpu().numpy(), T1.cpu().numpy()
        assert np.linalg.norm(w - w1) <= 1e-6 * np.linalg.norm(w1)
        assert np.linalg.norm(t - t1) <= 1e-6 * np.linalg.norm(t1)
    assert L.device_status() == 0


@pytest.mark.gpu
def test_batch_against_oracle():
    """Three lengths (Npad 8192, 16384, 32768), Morlet mu=6: the float32 bars
    against the float64 oracle."""
    _gpu()
    from ssqueezepy_b200._batch import SsqCwtBatch
    from oracle import ssq_oracle as O
    from tests._cases import rel_l2
    lengths = [4096, 6000, 12000]
    rng = np.random.default_rng(11)
    xs = [S.chirp_mix(N, rng).astype(np.float32) for N in lengths]
    plan = SsqCwtBatch(lengths, wavelet=('morlet', {'mu': 6.}))
    outs = plan(xs)
    for i, (x, (Tx, Wx, f, sc)) in enumerate(zip(xs, outs)):
        To, Wo, _ = O.ssq_cwt(x.astype(np.float64), 'morlet', (6.,), plan.scales64[i],
                              f[::-1].copy(), plan.weights64[i])
        assert rel_l2(Wx.cpu().numpy(), Wo) <= 1e-5
        assert rel_l2(Tx.cpu().numpy(), To) <= 1e-4


@pytest.mark.gpu
def test_batch_graph_replay_repeats_eager():
    torch = _gpu()
    from ssqueezepy_b200._batch import SsqCwtBatch
    rng = np.random.default_rng(3)
    xs = [S.chirp_mix(N, rng).astype(np.float32) for N in LENGTHS[:5]]
    eager = SsqCwtBatch(LENGTHS[:5], wavelet=('morlet', {'mu': 6.}))
    ref = [(t.clone(), w.clone()) for t, w, _, _ in eager(xs)]
    plan = SsqCwtBatch(LENGTHS[:5], wavelet=('morlet', {'mu': 6.}), graph=True)
    for _ in range(3):  # eager, capture + replay, replay
        plan.Tx.zero_()
        outs = plan(xs)
        torch.cuda.synchronize()
        for (t, w, _, _), (t0, w0) in zip(outs, ref):
            assert torch.equal(t, t0) and torch.equal(w, w0)
    assert plan._graph is not None
    assert plan.launches >= 1 + 2 * 3


@pytest.mark.gpu
def test_batch_autotune_picks_a_budget_and_keeps_results():
    torch = _gpu()
    from ssqueezepy_b200._batch import SsqCwtBatch
    rng = np.random.default_rng(9)
    xs = [S.chirp_mix(N, rng).astype(np.float32) for N in LENGTHS]
    ref = [(t.clone(), w.clone()) for t, w, _, _ in
           SsqCwtBatch(LENGTHS, wavelet=('morlet', {'mu': 6.}))(xs)]
    plan = SsqCwtBatch(LENGTHS, wavelet=('morlet', {'mu': 6.}), autotune=True, graph=True)
    assert plan.tuning and all(t['ms'] for t in plan.tuning)
    first = None
    for _ in range(2):
        outs = plan(xs)
        torch.cuda.synchronize()
        # the tuned band bound may send other rows through the band pass: the
        # same float64 transform summed in another order, so equal to float32
        # rounding, and replays of the tuned plan equal each other exactly
        for (t, w, _, _), (t0, w0) in zip(outs, ref):
            assert (w - w0).norm() <= 1e-7 * w0.norm()
            assert (t - t0).norm() <= 1e-6 * t0.norm()
        cur = [(t.clone(), w.clone()) for t, w, _, _ in outs]
        if first is not None:
            assert all(torch.equal(a, b) and torch.equal(c, d)
                       for (a, c), (b, d) in zip(cur, first))
        first = cur
    assert all('band_bins' in t for t in plan.tuning)
    assert L.device_status() == 0


@pytest.mark.gpu
def test_full_uneven_batch_every_signal_against_oracle():
    """The batched workload itself: 256 chirp mixtures with lengths uniform in
    [4096, 65536] (seed 1234), Morlet mu=6, one plan replayed as a CUDA graph.
    Every signal's Tx and Wx against the float64 oracle (the oracle runs the
    signals in parallel threads); max and median are printed."""
    torch = _gpu()
    from concurrent.futures import ThreadPoolExecutor
    from ssqueezepy_b200._batch import SsqCwtBatch
    from oracle import ssq_oracle as O
    from tests._cases import rel_l2
    xs = [x.astype(np.float32) for x in S.uneven_batch(256, 4096, 65536, 1234)]
    plan = SsqCwtBatch([len(x) for x in xs], wavelet=('morlet', {'mu': 6.}), graph=True)
    outs = plan(xs)
    torch.cuda.synchronize()

    def one(i):
        t, w, f, _ = outs[i]
        Tx, Wx = t.cpu().numpy(), w.cpu().numpy()
        To, Wo, _ = O.ssq_cwt(xs[i].astype(np.float64), 'morlet', (6.,), plan.scales64[i],
                              f[::-1].copy(), plan.weights64[i], gamma=10 * O.EPS32)
        return rel_l2(Wx, Wo), rel_l2(Tx, To)

    with ThreadPoolExecutor(4) as ex:
        errs = np.array(list(ex.map(one, range(len(xs)))))
    print(f'\n256 signals: Wx rel-L2 max {errs[:, 0].max():.2e} median '
          f'{np.median(errs[:, 0]):.2e}; Tx rel-L2 max {errs[:, 1].max():.2e} '
          f'median {np.median(errs[:, 1]):.2e}')
    assert errs[:, 0].max() <= 1e-5
    assert errs[:, 1].max() <= 1e-4
    assert L.device_status() == 0


@pytest.mark.gpu
def test_batch_band_pass_equals_tile_passes():
    """Rows whose wavelet band fits 512 bins take the band-limited single pass
    (ssqb_cwt_batch_ex); with it switched off every row takes the tile
    passes. Both compute in float64, so Wx agrees to float32 rounding and the
    bins agree except at exact ties."""
    torch = _gpu()
    from ssqueezepy_b200._batch import SsqCwtBatch
    rng = np.random.default_rng(21)
    lengths = [5000, 9000, 20000, 33000, 60000]
    xs = [S.chirp_mix(N, rng).astype(np.float32) for N in lengths]
    plan = SsqCwtBatch(lengths, wavelet=('morlet', {'mu': 6.}))
    assert any(g['band'][0] < (1 << 30) for g in plan.groups)
    band = [(t.clone(), w.clone()) for t, w, _, _ in plan(xs)]
    idx_band = plan.idx.clone()
    for g in plan.groups:
        g['band'] = (1 << 30, 0)
    tile = [(t.clone(), w.clone()) for t, w, _, _ in plan(xs)]
    torch.cuda.synchronize()
    for (t1, w1), (t0, w0) in zip(band, tile):
        assert (w1 - w0).norm() <= 1e-7 * w0.norm()
        assert (t1 - t0).norm() <= 1e-6 * t0.norm()
    assert int((idx_band != plan.idx).sum()) <= 2
    assert L.device_status() == 0
