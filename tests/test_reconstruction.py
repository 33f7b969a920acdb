# -*- coding: utf-8 -*-
"""Reconstruction properties, the reference's own self-consistency tests for
the path (tests/reconstruction_test.py), on the GPU: transform -> inverse
returns the signal within the reference's thresholds on its test-signal
families (exponential and linear chirps, fast frequency transitions, low and
high frequencies). The metric is mean |x - xrec| / rms(x)
(reconstruction_test.py:28-31). The STFT cases take the reference's n_fft
of 120 and 121 (through the chirp-z kernels) and 128."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as sb
    return sb


def _t(lo, hi, N):
    return np.linspace(lo, hi, N, endpoint=False)


def cos_f(freqs, N=128):
    """Adjacent segments of N samples, one cosine of frequency f per segment."""
    return np.concatenate([np.cos(2 * np.pi * f * _t(i, i + 1, N))
                           for i, f in enumerate(freqs)])


def mad_rms(x, xrec):
    return np.mean(np.abs(x - xrec)) / np.sqrt(np.mean(x ** 2))


def echirp(N):
    t = _t(0, 10, N)
    return np.cos(2 * np.pi * 3 * np.exp(t / 3)), t


def lchirp(N):
    t = _t(0, 10, N)
    return np.cos(np.pi * t ** 2), t


def _freqs(N, freqs):
    x = cos_f(freqs, N // len(freqs))
    return x, _t(0, len(x) / N, len(x))


def fast_transitions(N):
    return _freqs(N, np.array([N / 100, N / 200, N / 3, N / 20, N / 3 - 1, N / 50,
                               N / 4, N / 150]) / 8)


def low_freqs(N):
    return _freqs(N, [.3, .3, 1, 1, 2, 2])


def high_freqs(N):
    return _freqs(N, np.array([N / 2, N / 2 - 1, N / 4, N / 3]) / 4)


SIGNALS = (echirp, lchirp, fast_transitions, low_freqs, high_freqs)
WAVELET = ('gmw', {'beta': 8, 'dtype': 'float64'})
TH = .1


@pytest.mark.parametrize('fn', SIGNALS, ids=[f.__name__ for f in SIGNALS])
@pytest.mark.parametrize('scales', ['log', 'log-piecewise', 'linear'])
def test_ssq_cwt_inverts(fn, scales):
    sb = _gpu()
    x, ts = fn(2048)
    if fn is low_freqs:
        if scales == 'linear':
            pytest.skip("the default 'linear' grid does not reach these frequencies")
        scales = scales + ':maximal'
    Tx, *_ = sb.ssq_cwt(x, WAVELET, scales=scales, nv=32, t=ts, astensor=False)
    xrec = sb.issq_cwt(Tx, WAVELET)
    err = mad_rms(x, np.asarray(xrec))
    assert err < TH, (err, fn.__name__, scales)


@pytest.mark.parametrize('fn', SIGNALS, ids=[f.__name__ for f in SIGNALS])
@pytest.mark.parametrize('l1_norm', [True, False])
def test_cwt_inverts(fn, l1_norm):
    sb = _gpu()
    x, ts = fn(2048)
    scales = 'log:maximal' if fn in (low_freqs, high_freqs) else 'log'
    kw = dict(wavelet=WAVELET, scales=scales, l1_norm=l1_norm, nv=32)
    Wx, *_ = sb.cwt(x, t=ts, astensor=False, **kw)
    xrec = sb.icwt(Wx, one_int=True, **kw)
    err = mad_rms(x, xrec)
    assert err < TH, (err, fn.__name__, l1_norm)


def test_log_piecewise_inverts_both_ways():
    sb = _gpu()
    x, ts = echirp(1024)
    Tx, Wx, f, sc = sb.ssq_cwt(x, 'gmw', scales='log-piecewise', t=ts, astensor=False)
    e1 = mad_rms(x, np.asarray(sb.issq_cwt(Tx, 'gmw')))
    e2 = mad_rms(x, sb.icwt(Wx, 'gmw', scales=sc))
    assert e1 < .02 and e2 < .02, (e1, e2)


def test_component_inversion():
    """A noisy amplitude-modulated chirp: inverting Tx over a hand-set linear
    band recovers the clean chirp (reconstruction_test.py:126-157 with the
    band of toolkit.lin_band, toolkit.py:7-20)."""
    sb = _gpu()
    N = 2048
    t = np.linspace(0, 10, N, False)
    xo = np.cos(2 * np.pi * np.exp(t / 3)) * (1 + .3 * cos_f([1], N))
    # the reference's noise: the legacy generator seeded with 4
    x = xo + np.sqrt(6.) * np.random.RandomState(4).standard_normal(N)
    wav = ('gmw', {'beta': 6})
    Tx, *_ = sb.ssq_cwt(x, wav, scales='log:maximal', nv=32, t=t, flipud=0,
                        astensor=False)
    na = Tx.shape[0]
    bw, slope, offset = .035, .44, .45
    Cs = (slope * (np.linspace(0, 1, N) + offset) * na).astype('int32')
    band = (bw * na * np.ones(N)).astype('int32')
    xrec = np.asarray(sb.issq_cwt(Tx, wav, Cs, band))[0]
    err_sig = mad_rms(xo, xrec)
    err_spc = mad_rms(np.abs(np.fft.rfft(xo)), np.abs(np.fft.rfft(xrec)))
    assert err_sig <= .40, err_sig
    assert err_spc <= .10, err_spc


@pytest.mark.parametrize('N', [128, 129])
@pytest.mark.parametrize('n_fft', [120, 121, 128])
@pytest.mark.parametrize('hop_len', [1, 2, 3])
@pytest.mark.parametrize('modulated', [True, False])
def test_stft_istft_inverts(N, n_fft, hop_len, modulated):
    sb = _gpu()
    x = np.random.default_rng(N + hop_len).standard_normal(N)
    kw = dict(hop_len=hop_len, n_fft=n_fft, modulated=modulated)
    Sx = sb.stft(x, dtype='float64', **kw)
    xr = sb.istft(Sx, N=len(x), **kw).cpu().numpy()
    assert len(xr) == N
    assert np.abs(x - xr).mean() < 1e-14


@pytest.mark.parametrize('N', [128, 129])
@pytest.mark.parametrize('n_fft', [120, 121])
@pytest.mark.parametrize('window_scaling', [1., .5])
def test_ssq_stft_inverts(N, n_fft, window_scaling):
    sb = _gpu()
    x = np.random.default_rng(N).standard_normal(N)
    window = None
    if window_scaling != 1:
        window = sb.get_window(None, win_len=n_fft, n_fft=n_fft) * window_scaling
    Tx, *_ = sb.ssq_stft(x, window=window, n_fft=n_fft, astensor=False)
    xr = np.asarray(sb.issq_stft(Tx, window=window, n_fft=n_fft))
    assert len(xr) == N
    assert np.abs(x - xr).mean() < .1
