# -*- coding: utf-8 -*-
"""Inverse synchrosqueezing, issq_cwt / issq_stft (ssqb_issq): full and
per-component inversion against ssqueezepy's own outputs on seeded complex
Tx (tests/golden/issq.npz, float64 wavelets), in float64 and float32."""
import ctypes
import os

import numpy as np
import pytest

from ssqueezepy_b200 import _lib as L
from ssqueezepy_b200 import _params as P
from tests._cases import rel_l2

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'issq.npz')


def _inputs():
    from tests.test_oracle import _issq_inputs
    return _issq_inputs()


def test_issq_rejects_bad_arguments():
    lib = L.load()
    p = ctypes.c_void_p(8)
    assert lib.ssqb_issq(None, 10, 10, None, None, 0, 1.0, 0, p, None) == L.EINVAL
    assert lib.ssqb_issq(p, 0, 10, None, None, 0, 1.0, 0, p, None) == L.EINVAL
    assert lib.ssqb_issq(p, 10, 10, None, None, 2, 1.0, 0, p, None) == L.EINVAL
    assert lib.ssqb_issq(p, 10, 10, p, p, 17, 1.0, 0, p, None) == L.EUNSUPPORTED
    assert lib.ssqb_issq(p, 10, 10, None, None, 0, 1.0, 7, p, None) == L.EINVAL


@pytest.mark.gpu
@pytest.mark.parametrize('dtype', [np.complex128, np.complex64])
def test_issq_matches_reference(dtype):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    Tc, Ts, cc, cw = _inputs()
    tol = 1e-12 if dtype == np.complex128 else 1e-6
    for key, wav in (('gmw', ('gmw', {'dtype': 'float64'})),
                     ('morlet6', ('morlet', {'mu': 6., 'dtype': 'float64'}))):
        x = sb.issq_cwt(Tc.astype(dtype), wav)
        assert isinstance(x, np.ndarray) and x.shape == (700,)
        assert rel_l2(x, g['cwt_full_' + key]) < tol
        xc = sb.issq_cwt(Tc.astype(dtype), wav, cc, cw)
        assert xc.shape == (3, 700) and xc.dtype == np.float64
        assert rel_l2(xc, g['cwt_comp_' + key]) < tol
    xs = sb.issq_stft(torch.as_tensor(Ts.astype(dtype), device='cuda'), 'hann', n_fft=256)
    assert isinstance(xs, torch.Tensor)
    assert rel_l2(xs.cpu().numpy(), g['stft_full_hann256']) < tol
    xsc = sb.issq_stft(Ts.astype(dtype), 'hann', cc=cc, cw=cw, n_fft=256)
    assert rel_l2(xsc, g['stft_comp_hann256']) < tol


@pytest.mark.gpu
def test_issq_cwt_reconstructs_the_signal():
    """ssq_cwt then issq_cwt gives back x up to the synchrosqueezing's own
    reconstruction error (4.3e-3 relative L2 for this signal in the float64
    oracle)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as sb
    from ssqueezepy_b200 import _signals as S
    x = S.chirp_tone(4096, seed=2)
    Tx, *_ = sb.ssq_cwt(x, ('gmw', {'dtype': 'float64'}), astensor=False)
    xr = sb.issq_cwt(Tx, ('gmw', {'dtype': 'float64'}))
    assert np.linalg.norm(xr - x) / np.linalg.norm(x) < 0.02  # 4.3e-3 in the oracle
