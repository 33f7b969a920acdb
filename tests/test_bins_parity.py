# -*- coding: utf-8 -*-
"""Bin-index parity of the CUDA path with the float64 oracle.

The fused CWT kernel writes a uint16 bin index per (row, column): the bin of
the phase transform w = |Im(dWx conj Wx)| / (|Wx|^2 2 pi) under the rule of
algos.py:859-953, 0xFFFF where |Wx| <= gamma. Here that index, read back
from `ssqb_cwt`, is compared entry by entry with the oracle's float64 bins
of the same float32 input (rounded to float32 first, then taken as float64
on both sides, so that input rounding is not counted as a difference).

The bar: bins bit-exact except where the float64 w lies within one float32
ulp of the rounding edge between the two bins; such entries are counted and
printed. Masks (|Wx| > gamma) must agree except within 1e-12 of gamma."""
import numpy as np
import pytest
import torch

from oracle import ssq_oracle as O
from ssqueezepy_b200 import _params as P
from ssqueezepy_b200 import _signals as S
from ssqueezepy_b200 import _transforms as T
from tests._cases import WAVS, chirp_signal, oracle_kind

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def sb():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as m
    m._lib.load()
    return m


def cuda_bins(x32, wk, scales, sqf, maprange='peak'):
    """Bin index and host parameters of the CUDA path for one float32 signal
    (the ssq_cwt defaults: reflect padding, flipud)."""
    nm, opts = WAVS[wk]
    wav = P.Wavelet((nm, dict(opts, dtype='float32')))
    N = len(x32)
    fp = T._ssq_plan(wav, scales, N, 32, sqf, maprange, 'reflect', 1.)
    na = T._scales_plan(scales, N, wav, 32)['na']
    r = T._cwt_core(torch.as_tensor(x32, device='cuda'), wav, scales, 32, None, None,
                    'reflect', False, False, False, want_idx=True,
                    ssq=(fp['mode'], fp['bp'], na, True))
    idx = r['idx'][0, :, :N].cpu().numpy()
    return idx, r['scales'], fp, r['gamma']


def check(x, wk, scales='log-piecewise', sqf=None):
    x32 = np.asarray(x, np.float32)
    idx, s64, fp, gamma = cuda_bins(x32, wk, scales, sqf)
    W, dW = O.cwt(x32.astype(np.float64), *oracle_kind(wk), s64)
    return O.bin_parity(idx, W, dW, fp['f_asc'], fp['mode'] != 2, True, gamma)


@pytest.mark.parametrize('N, wk, sqf', [(10000, 'morlet6', 'log'),
                                        (160000, 'gmw3_60', None)])
def test_bins_match_float64_oracle_full_size(sb, N, wk, sqf):
    """The N=10,000 Morlet (log bins) and N=160,000 GMW (log-piecewise bins)
    single-signal workloads."""
    rep = check(chirp_signal(N, seed=0), wk, sqf=sqf)
    print(f'\nbins N={N} {wk}: {rep}')
    assert rep['kept'] > 0.9 * rep['entries']
    assert rep['other'] == 0, rep
    assert rep['mask_other'] == 0, rep


@pytest.mark.parametrize('seed', [0, 1])
def test_bins_match_float64_oracle_chirp_mixtures(sb, seed):
    """Chirp mixtures (the batched workload's signal family), Morlet, at a
    short and a long length."""
    for N in (4096 + 1237 * seed, 65536 - 999 * seed):
        x = S.chirp_mix(N, np.random.default_rng(100 + seed))
        rep = check(x, 'morlet6')
        print(f'\nbins mixture N={N}: {rep}')
        assert rep['other'] == 0, rep
        assert rep['mask_other'] == 0, rep
