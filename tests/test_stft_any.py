# -*- coding: utf-8 -*-
"""STFT and ssq_stft for n_fft that are not powers of two (Bluestein's
chirp-z transform inside the fused STFT kernel), against the reference's
outputs (tests/golden/stft_any.npz, made by tests/golden/make_golden.py):
odd and even lengths, the reference's own benchmark length 598, modulated
on and off."""
import os

import numpy as np
import pytest

from tests._cases import rel_l2
from tests.golden.make_golden import STFT_ANY_CASES

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'stft_any.npz')
IDS = [c[0] for c in STFT_ANY_CASES]


def test_stft_any_argument_checks():
    import ssqueezepy_b200 as sb
    with pytest.raises(NotImplementedError):
        sb.stft(np.zeros(5000), n_fft=1500)   # not a power of two, above 1024


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as sb
    return sb


@pytest.mark.gpu
@pytest.mark.parametrize('case', STFT_ANY_CASES, ids=IDS)
def test_stft_any_length_matches_reference(case):
    sb = _gpu()
    name, N, n_fft, hop, mod, win = case
    g = np.load(GOLD)
    x = g[name + '/x']
    Sx, dSx = sb.stft(x, win, n_fft=n_fft, hop_len=hop, modulated=mod, derivative=True,
                      dtype='float64')
    assert tuple(Sx.shape) == g[name + '/Sx'].shape
    assert rel_l2(Sx.cpu().numpy(), g[name + '/Sx']) <= 1e-11
    assert rel_l2(dSx.cpu().numpy(), g[name + '/dSx']) <= 1e-11
    Tx, *_ = sb.ssq_stft(x, win, n_fft=n_fft, hop_len=hop, modulated=mod, dtype='float64',
                         astensor=False)
    assert rel_l2(Tx, g[name + '/Tx']) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize('case', STFT_ANY_CASES, ids=IDS)
def test_stft_any_length_float32(case):
    sb = _gpu()
    name, N, n_fft, hop, mod, win = case
    g = np.load(GOLD)
    Sx = sb.stft(g[name + '/x'].astype(np.float32), win, n_fft=n_fft, hop_len=hop,
                 modulated=mod, dtype='float32')
    assert Sx.dtype.is_complex and Sx.element_size() == 8
    assert rel_l2(Sx.cpu().numpy(), g[name + '/Sx']) <= 1e-6


@pytest.mark.gpu
def test_default_n_fft_of_a_short_signal():
    """N = 300 < 512: the default n_fft is N itself (_stft.py:120), which
    is not a power of two: computed, not refused."""
    sb = _gpu()
    x = np.random.default_rng(0).standard_normal(300)
    Sx = sb.stft(x, dtype='float64')
    assert Sx.shape[0] == 300 // 2 + 1
    Tx, *_ = sb.ssq_stft(x, dtype='float64')
    assert np.isfinite(Tx.cpu().numpy()).all()


@pytest.mark.gpu
@pytest.mark.parametrize('n_fft', [513, 600, 640])
def test_stft_mixed_radix_lengths_match_oracle(n_fft):
    """n_fft 513-640: the chirp-z convolution runs at the mixed-radix length
    1280 = 5 x 4^4 instead of 2048. Sx, dSx against the float64 oracle, hop
    1 and 3 (the reference's benchmark length 598 is in the golden cases)."""
    sb = _gpu()
    from oracle import ssq_oracle as O
    from ssqueezepy_b200 import _params as P
    x = np.random.default_rng(n_fft).standard_normal(2500)
    win, dwin = P.get_window('hann', n_fft, n_fft, derivative=True)
    for hop in (1, 3):
        Sx, dSx = sb.stft(x, 'hann', n_fft=n_fft, hop_len=hop, derivative=True,
                          dtype='float64')
        So, dSo = O.stft(x, win, dwin, n_fft, hop=hop)
        assert rel_l2(Sx.cpu().numpy(), So) <= 1e-11, (n_fft, hop)
        assert rel_l2(dSx.cpu().numpy(), dSo) <= 1e-11, (n_fft, hop)
