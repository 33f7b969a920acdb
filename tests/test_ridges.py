# -*- coding: utf-8 -*-
"""extract_ridges on the GPU (ssqb_extract_ridges) against ssqueezepy's own
outputs (tests/golden/ridges.npz: serial code path, float64 and float32,
log and linear frequency axes, one and two ridges)."""
import ctypes
import os

import numpy as np
import pytest

from ssqueezepy_b200 import _lib as L

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'ridges.npz')


def test_ridges_reject_bad_arguments():
    lib = L.load()
    p = ctypes.c_void_p(8)
    assert lib.ssqb_extract_ridges(None, 10, 10, p, p, 2., 1, 4, 1e-7, 0, p, None, None, p,
                                   1 << 20, None) == L.EINVAL
    assert lib.ssqb_extract_ridges(p, 10, 10, p, p, 2., 0, 4, 1e-7, 0, p, None, None, p,
                                   1 << 20, None) == L.EINVAL
    assert lib.ssqb_extract_ridges(p, 10, 10, p, p, 2., 1, 4, 1e-7, 0, p, None, None, p,
                                   16, None) == L.EWORKSPACE
    assert lib.ssqb_extract_ridges(p, 40000, 10, p, p, 2., 1, 4, 1e-7, 0, p, None, None, p,
                                   1 << 30, None) == L.EUNSUPPORTED
    assert lib.ssqb_ridges_workspace_bytes(64, 400, L.F32) == 3 * 64 * 400 * 4 + 400 * 4


@pytest.mark.gpu
@pytest.mark.parametrize('dt', ['f64', 'f32'])
@pytest.mark.parametrize('ax, tr', [('log', 'cwt'), ('lin', 'stft')])
@pytest.mark.parametrize('nr, bw', [(1, 15), (2, 4)])
def test_ridges_match_reference(dt, ax, tr, nr, bw):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as sb
    g = np.load(GOLD)
    T = g['Tf'] if dt == 'f64' else g['Tf'].astype(np.complex64)
    key = '%s_%s_r%d' % (dt, ax, nr)
    i, f, e = sb.extract_ridges(T, g['scales_' + ax], penalty=2., n_ridges=nr, bw=bw,
                                transform=tr, get_params=True)
    assert np.array_equal(i, g[key + '_idx'])
    assert np.array_equal(f, g[key + '_f'])
    assert np.allclose(e, g[key + '_e'], rtol=1e-6 if dt == 'f32' else 1e-13)
    assert L.device_status() == 0
