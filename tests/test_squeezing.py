# -*- coding: utf-8 -*-
"""`squeezing` other than 'sum' (ssqueezing.py:196-201): the squeeze sums
ones / len(Wx) ('lebesgue'), |Wx| ('abs') or squeezing(Wx) (a function); with
no phase transform given, the reference takes the phase from those values and
dWx, and so does this package. Against the reference's outputs
(tests/golden/squeezing.npz, made by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from tests._cases import rel_l2
from tests.golden.make_golden import square

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'squeezing.npz')
W64 = ('gmw', {'dtype': 'float64'})
CASES = [('lebesgue', 'lebesgue'), ('abs', 'abs'), ('square', square)]


def test_squeezing_argument_checks():
    import ssqueezepy_b200 as sb
    with pytest.raises(ValueError):
        sb.ssq_cwt(np.zeros(64), squeezing='max')
    with pytest.raises(TypeError):
        sb.ssq_cwt(np.zeros(64), squeezing=3)


def test_squeeze_values_rules():
    import torch
    from ssqueezepy_b200._transforms import _squeeze_values
    W = torch.tensor([[3 + 4j, 1j], [0j, -2 + 0j]], dtype=torch.complex128)
    assert torch.equal(_squeeze_values(W, 'sum'), W)
    assert torch.equal(_squeeze_values(W, 'abs'),
                       torch.tensor([[5, 1], [0, 2]], dtype=torch.complex128))
    assert torch.equal(_squeeze_values(W, 'lebesgue'), torch.full_like(W, 0.5))
    assert torch.equal(_squeeze_values(W, square), W * W)
    with pytest.raises(ValueError):
        _squeeze_values(W, lambda a: a[0])


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')


@pytest.mark.gpu
@pytest.mark.parametrize('name, sqz', CASES, ids=[c[0] for c in CASES])
def test_ssq_cwt_squeezing_matches_reference(name, sqz):
    _gpu()
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    Tx, *_ = sb.ssq_cwt(g['x'], W64, nv=8, squeezing=sqz, astensor=False)
    assert rel_l2(Tx, g['cwt_%s/Tx' % name]) <= 1e-9
    Tx, *_ = sb.ssq_cwt(g['x'], W64, nv=8, squeezing=sqz, get_w=True, astensor=False)
    assert rel_l2(Tx, g['cwt_%s_w/Tx' % name]) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize('name, sqz', CASES, ids=[c[0] for c in CASES])
def test_ssq_stft_squeezing_matches_reference(name, sqz):
    _gpu()
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    Tx, *_ = sb.ssq_stft(g['x'], 'hann', n_fft=64, squeezing=sqz, dtype='float64',
                         astensor=False)
    assert rel_l2(Tx, g['stft_%s/Tx' % name]) <= 1e-9


@pytest.mark.gpu
def test_ssqueeze_squeezing_abs_equals_ssq_cwt():
    """The public ssqueeze with squeezing='abs' on ssq_cwt's own Wx, dWx."""
    _gpu()
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    Tx0, Wx, f, sc, dWx = sb.ssq_cwt(g['x'], W64, nv=8, squeezing='abs', get_dWx=True)
    Tx, _ = sb.ssqueeze(Wx, None, ssq_freqs=None, scales=sc, squeezing='abs',
                        maprange='peak', wavelet=W64, gamma=10 * np.finfo(np.float64).eps,
                        dWx=dWx, flipud=True)
    assert rel_l2(Tx.cpu().numpy(), Tx0.cpu().numpy()) <= 1e-12


@pytest.mark.gpu
def test_phase_transform_without_bins_leaves_status_clean():
    """w requested without a bin index (the squeeze then bins w itself):
    no bin decisions are made in the transform, so none is flagged."""
    _gpu()
    import ssqueezepy_b200 as sb
    from ssqueezepy_b200 import _lib as L
    g = np.load(GOLD)
    L.device_status()
    sb.ssq_cwt(g['x'], W64, nv=8, squeezing='abs', get_w=True)
    sb.ssq_stft(g['x'], 'hann', n_fft=64, squeezing='abs', get_w=True, dtype='float64')
    assert L.device_status() == 0
