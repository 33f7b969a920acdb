# -*- coding: utf-8 -*-
"""Properties the reference's own test suite checks on this path, restated
for this package (tests/fft_test.py, tests/z_all_test.py,
tests/ridge_extraction_test.py): the two squeeze forms agree, batched input
equals per-signal calls, float32 and float64 paths agree, output dtypes,
trigdiff equals the CWT's own derivative, the log-piecewise split, and the
ridge examples. Where the reference compares its CPU and GPU back ends, the
comparison here is between this package's routes to the same result."""
import numpy as np
import pytest

from ssqueezepy_b200 import _lib as L
from ssqueezepy_b200 import _params as P


#### CPU #####################################################################
def test_logscale_transition_idx():
    """A log grid whose tail keeps every 2nd / 3rd / 4th value splits where
    the spacing changes (z_all_test.py:368-380)."""
    scales = np.exp(np.linspace(0, 5, 512))
    idx = 399
    for step in (2, 3, 4):
        scales = np.hstack([scales[:idx], scales[idx + step - 1::step]])
        assert P.logscale_transition_idx(scales) == idx, step


def test_check_ssqueezing_args():
    """Bad arguments raise as in the reference (z_all_test.py:439-453)."""
    from ssqueezepy_b200._transforms import _check_ssq_args
    with pytest.raises(ValueError):
        _check_ssq_args('sum', 'peak', 'numeric', get_w=False)
    with pytest.raises(ValueError):
        _check_ssq_args('sum', 'peak', 'numeric', get_w=True, difforder=3)
    with pytest.raises(TypeError):
        _check_ssq_args('sum', 5, 'trig')
    with pytest.raises(ValueError):
        _check_ssq_args('sum', ('a', 1), 'trig')
    with pytest.raises(ValueError):
        _check_ssq_args('max', 'peak', 'trig')


#### GPU #####################################################################
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as sb
    return sb, torch


def _ssq_freqs(n, scaletype):
    if scaletype == 'log-piecewise':
        a = np.logspace(-3, -1, n // 2, base=2.)
        b = np.logspace(np.log2(a[-1]) + .5, 0, n - n // 2, base=2.)
        return np.hstack([a, b])
    if scaletype == 'log':
        return np.logspace(-6, -.2, n, base=2.)
    return np.linspace(1e-3, .5, n)


@pytest.mark.gpu
@pytest.mark.parametrize('dtype', ['float32', 'float64'])
@pytest.mark.parametrize('scaletype', ['log-piecewise', 'log', 'linear'])
@pytest.mark.parametrize('flipud', [False, True])
def test_ssqueeze_equals_indexed_sum(dtype, scaletype, flipud):
    """The squeeze taking the phase from (Wx, dWx) and the squeeze of a
    given w agree (fft_test.py:351-377, its thresholds)."""
    _, torch = _gpu()
    rng = np.random.default_rng(0)
    gamma = 1e-2
    Wx = (rng.standard_normal((100, 512)).astype(dtype) * (1 + 2j))
    dWx = (rng.standard_normal((100, 512)).astype(dtype) * (2 - 1j))
    w = np.abs((dWx / Wx).imag / (2 * np.pi))
    w[np.abs(Wx) < gamma] = np.inf
    f = _ssq_freqs(len(Wx), scaletype)
    logscale = scaletype.startswith('log')
    mode, bp = P.bin_params(f, logscale)
    const = np.full(len(Wx), np.log(2) / 32) if logscale else f
    dev = torch.device('cuda')
    Wd, dWd = torch.as_tensor(Wx, device=dev), torch.as_tensor(dWx, device=dev)
    wd = torch.as_tensor(w, device=dev)
    cd = torch.as_tensor(const, dtype=torch.float64, device=dev)
    prec = L.F64 if dtype == 'float64' else L.F32
    cb = L.make_bins(mode, bp, len(Wx), flipud)
    out0, out1 = torch.empty_like(Wd), torch.empty_like(Wd)
    lib = L.load()
    L.check(lib.ssqb_indexed_sum(L.ptr(Wd), L.ptr(wd), L.ptr(cd), cb, 1, 100, 512, prec,
                                 L.ptr(out0), L.stream_ptr()))
    L.check(lib.ssqb_ssqueeze_fast(L.ptr(Wd), L.ptr(dWd), None, L.ptr(cd), cb, gamma, 1,
                                   100, 512, prec, L.ptr(out1), L.stream_ptr()))
    adiff = (out0 - out1).abs().mean().item()
    th = ((1e-16 if dtype == 'float64' else 1e-8) if logscale else
          (1e-13 if dtype == 'float64' else 1e-5))
    assert adiff < th, adiff


@pytest.mark.gpu
@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_ssq_cwt_batched_equals_per_signal(dtype):
    """2D x gives each row's own ssq_cwt (fft_test.py:559-597)."""
    sb, _ = _gpu()
    x = np.random.default_rng(0).standard_normal((4, 256))
    wav = ('gmw', {'dtype': dtype})
    Tx0, Wx0, *_ = sb.ssq_cwt(x, wav, astensor=False)
    for i in range(4):
        Tx, Wx, *_ = sb.ssq_cwt(x[i], wav, astensor=False)
        assert np.allclose(Wx, Wx0[i]) and np.allclose(Tx, Tx0[i]), i


@pytest.mark.gpu
def test_ssq_stft_batched_equals_per_signal():
    """fft_test.py:599-632 for the STFT."""
    sb, _ = _gpu()
    x = np.random.default_rng(1).standard_normal((4, 256))
    Tx0, Sx0, *_ = sb.ssq_stft(x, n_fft=64, astensor=False)
    for i in range(4):
        Tx, Sx, *_ = sb.ssq_stft(x[i], n_fft=64, astensor=False)
        assert np.allclose(Sx, Sx0[i]) and np.allclose(Tx, Tx0[i]), i


@pytest.mark.gpu
def test_higher_order_float32_tracks_float64():
    """order=range(3) at float32 against float64 within the reference's
    float32 threshold (fft_test.py:514-536)."""
    sb, _ = _gpu()
    t = np.linspace(0, 1, 256, endpoint=False)
    x = np.cos(2 * np.pi * (10 * t + 40 * t ** 2))
    x += x[::-1]
    outs = [sb.ssq_cwt(x, ('gmw', {'dtype': d}), order=range(3), astensor=False)
            for d in ('float32', 'float64')]
    assert np.abs(outs[0][0] - outs[1][0]).mean() < 1e-4
    assert np.abs(outs[0][1] - outs[1][1]).mean() < 1e-4


@pytest.mark.gpu
def test_output_dtypes():
    """float32 / complex64 outputs for a float32 wavelet, float64 /
    complex128 for float64, ssq_freqs float64 either way, also with
    order=2 (z_all_test.py:383-413)."""
    sb, torch = _gpu()
    x = np.random.default_rng(2).standard_normal(256)
    names = ('Tx', 'Wx', 'ssq_freqs', 'scales')
    for dt, kw in (('float32', {}), ('float32', dict(order=2)), ('float64', {})):
        outs = dict(zip(names, sb.ssq_cwt(x, ('gmw', {'dtype': dt}), astensor=False,
                                          **kw)))
        for k, v in outs.items():
            if k == 'ssq_freqs':
                assert v.dtype == np.float64, (dt, k)
            elif dt == 'float32':
                assert v.dtype in (np.float32, np.complex64), (dt, k, v.dtype)
            else:
                assert v.dtype in (np.float64, np.complex128), (dt, k, v.dtype)


@pytest.mark.gpu
@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_trigdiff_equals_cwt_derivative(dtype):
    """z_all_test.py:352-365 with its thresholds: trigdiff of the padded
    transform against the transform's own derivative."""
    sb, _ = _gpu()
    N = 256
    x = np.random.default_rng(3).standard_normal(N)
    wav = ('gmw', {'dtype': dtype})
    Wx, _, dWx = sb.cwt(x, wav, derivative=True, rpadded=True, astensor=False)
    _, n1, _ = P.p2up(N)
    dWx2 = sb.trigdiff(Wx, rpadded=True, N=N, n1=n1)
    mae = np.mean(np.abs(dWx[:, n1:n1 + N] - dWx2))
    assert mae < (1e-15 if dtype == 'float64' else 1e-7), mae


@pytest.mark.gpu
def test_ridge_basic_example():
    """The 3x3 example of ridge_extraction_test.py:17-26 (after MATLAB's
    wsstridge documentation): integer input, ridge along the last row."""
    sb, _ = _gpu()
    m = np.array([[1, 4, 4], [2, 2, 2], [5, 5, 4]])
    idx, *_ = sb.extract_ridges(m, np.exp([1, 2, 3]), penalty=2.0, get_params=True)
    assert np.allclose(idx, np.array([[2, 2, 2]]))


@pytest.mark.gpu
def test_ridges_of_all_four_transforms():
    """Cubic-polynomial sweep plus a pure tone through cwt / ssq_cwt / stft /
    ssq_stft ridges with padtype 'wrap' (ridge_extraction_test.py:29-87):
    shapes and bounds, and the two-ridge split holding the tone (constant
    row) and the sweep apart. The STFTs take n_fft=256: the default here would
    be N=257, and this package's STFT takes powers of two."""
    sb, _ = _gpu()
    N, f = 257, 0.5
    t = np.linspace(0, 10, N, endpoint=True)
    phase = 2 * np.pi * (0.025 * t ** 4 / 4 - 0.36 * t ** 3 / 3 + 1.25 * t ** 2 / 2 + 2 * t)
    x = np.cos(phase) + np.sin(2 * np.pi * f * t)
    Twx, Wx, fc, scales = sb.ssq_cwt(x, 'morlet', t=t, padtype='wrap', astensor=False)
    Tsx, Sx, fs_, Sfs = sb.ssq_stft(x, None, n_fft=256, fs=1 / (t[1] - t[0]),
                                    padtype='wrap', astensor=False)
    kw = dict(penalty=2.0, n_ridges=2)
    for Tf, axis, tr, bw in ((Wx, scales, 'cwt', 15), (Twx, fc, 'cwt', 4),
                             (Sx, Sfs, 'stft', 4), (Tsx, fs_, 'stft', 4)):
        r = sb.extract_ridges(Tf, axis, transform=tr, bw=bw, **kw)
        assert r.shape == (Tf.shape[1], 2)
        assert r.min() >= 0 and r.max() < Tf.shape[0]
        # the tone holds one ridge near a fixed row
        assert min(np.std(r[:, 0]), np.std(r[:, 1])) < 0.05 * Tf.shape[0], tr
