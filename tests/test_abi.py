# -*- coding: utf-8 -*-
"""The C-ABI library loads, exports every symbol include/ssqb.h declares, and
rejects bad arguments before touching a device (no GPU needed)."""
import ctypes
import os
import re

import pytest

from ssqueezepy_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, 'include', 'ssqb.h')).read()
    return sorted(set(re.findall(r'SSQB_API\s+[\w\s\*]+?\b(ssqb_\w+)\s*\(', src)))


def test_header_declares_entry_points():
    names = _declared()
    assert 'ssqb_cwt' in names and 'ssqb_squeeze' in names and 'ssqb_stft' in names
    assert set(names) == set(L.SIGNATURES), (names, sorted(L.SIGNATURES))


def test_library_exports_all_symbols():
    lib = L.load()
    for name in _declared():
        assert hasattr(lib, name), name
    assert lib.ssqb_version() >= 1


def _cwt_call(**kw):
    lib = L.load()
    a = dict(x=ctypes.c_void_p(8), B=1, N=100, Npad=256, n1=78, padtype=1, rpadded=0,
             scales=ctypes.c_void_p(8), na=10, wav=L.make_wavelet(0, (6., 1e-8, 1., 0.)),
             dt=1.0, bins=None, gamma=1e-6, prec=0, Wx=ctypes.c_void_p(8), dWx=None,
             w=None, idx=None, ipitch=0, ws=ctypes.c_void_p(8), wsb=1 << 30, st=None)
    a.update(kw)
    return lib.ssqb_cwt(a['x'], a['B'], a['N'], a['Npad'], a['n1'], a['padtype'],
                        a['rpadded'], a['scales'], a['na'], a['wav'], a['dt'],
                        a['bins'], a['gamma'], a['prec'], a['Wx'], a['dWx'], a['w'],
                        a['idx'], a['ipitch'], a['ws'], a['wsb'], a['st'])


@pytest.mark.parametrize('kw, code', [
    (dict(B=0), L.EINVAL),
    (dict(N=0), L.EINVAL),
    (dict(Npad=300), L.EUNSUPPORTED),
    (dict(Npad=1 << 23), L.EUNSUPPORTED),
    (dict(n1=200), L.EINVAL),
    (dict(padtype=9), L.EINVAL),
    (dict(prec=3), L.EINVAL),
    (dict(idx=ctypes.c_void_p(8), ipitch=50,
          bins=L.make_bins(0, (0., 0.1, 0, 0, 0), 10, 1)), L.EINVAL),
    (dict(dt=0.0), L.EINVAL),
    (dict(x=None), L.EINVAL),
    (dict(Wx=None), L.EINVAL),
    (dict(wsb=16), L.EWORKSPACE),
    (dict(wav=L.make_wavelet(7, (0, 0, 0, 0))), L.EINVAL),
    (dict(wav=L.make_wavelet(0, (6., 1e-8, 1., 0.), kc=[1., 2.])), L.EINVAL),
    (dict(wav=L.make_wavelet(1, (3., 60., 1., 0.), kc=[1.] * 9)), L.EINVAL),
    (dict(wav=L.make_wavelet(1, (3., 60., 1., 0.), kc=[1., float('nan')])), L.EINVAL),
    (dict(idx=ctypes.c_void_p(8), bins=None), L.EINVAL),
    (dict(idx=ctypes.c_void_p(8), bins=L.make_bins(0, (0., 0.1, 0, 0, 0), 11, 1)),
     L.EINVAL),
])
def test_cwt_rejects_bad_arguments(kw, code):
    assert _cwt_call(**kw) == code
    assert L.load().ssqb_last_error()


def test_other_entry_points_reject_bad_arguments():
    lib = L.load()
    p = ctypes.c_void_p(8)
    assert lib.ssqb_squeeze(p, p, 0, p, 0, 10, 10, 10, 0, p, None) == L.EINVAL
    assert lib.ssqb_squeeze(p, p, 0, p, 1, 10, 10, 70000, 0, p, None) == L.EINVAL
    assert lib.ssqb_squeeze(p, p, 0, p, 1, 10, 10, 10000, 0, p, None) == L.EUNSUPPORTED
    assert lib.ssqb_squeeze(p, p, 5, p, 1, 10, 10, 10, 0, p, None) == L.EINVAL
    assert lib.ssqb_ssqueeze_fast(p, p, None, p, None, 1e-6, 1, 5, 5, 0, p, None) \
        == L.EINVAL
    b = L.make_bins(2, (0., 0.1, 0, 0, 0), 65, 0)
    # lengths past the chirp-z range (not a power of two and above 1024, or
    # below 4) are refused before any device work
    for n_fft in (1025, 2000, 3):
        assert lib.ssqb_stft(p, 1, 100, n_fft, 1, 50, 1, 1, p, p, p, b, 1e-6, 0, p, None,
                             None, None, 0, None) == L.EUNSUPPORTED, n_fft
    assert lib.ssqb_stft(p, 1, 100, 128, 0, 64, 1, 1, p, p, p, b, 1e-6, 0, p, None,
                         None, None, 0, None) == L.EINVAL
    assert lib.ssqb_icwt(None, p, None, 1.0, 1, 10, 10, 0, p, None) == L.EINVAL


def test_workspace_query():
    lib = L.load()
    small = lib.ssqb_cwt_workspace_bytes(1, 100, 256, 50, 0)
    assert small == 256 * 16  # spectrum only: one pass
    big = lib.ssqb_cwt_workspace_bytes(1, 160000, 1 << 18, 293, 0)
    assert big >= (1 << 18) * 16 + 2 * (1 << 18) * 8
    assert lib.ssqb_cwt_workspace_bytes(0, 1, 1, 1, 0) == 0


def test_transform_raises_without_cuda(monkeypatch):
    import numpy as np
    import torch
    import ssqueezepy_b200 as sb
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        sb.ssq_cwt(np.random.randn(64))
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        sb.stft(np.random.randn(64))
