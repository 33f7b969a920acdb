# -*- coding: utf-8 -*-
"""The band-limited single pass of `ssqb_cwt_ex`: rows whose wavelet band
spans at most a quarter of a transform tile skip the four-step of the full
padded length. Its outputs must equal the tile passes' (`ssqb_cwt`, the same
call without host scales) to rounding: float64 arithmetic differs only in
the order of the sums, so Wx agrees to ~1e-15 and the bins agree except at
exact ties; float32 arithmetic to its own rounding."""
import numpy as np
import pytest
import torch

from ssqueezepy_b200 import _lib as L
from ssqueezepy_b200 import _params as P
from ssqueezepy_b200 import _signals as S
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu

CASES = [  # (N, B, wavelet, precision): two-pass lengths with narrow rows
    (160000, 1, ('gmw', {'gamma': 3., 'beta': 60.}), 'F32X'),
    (10000, 3, ('morlet', {'mu': 6.}), 'F32X'),
    (10000, 2, ('morlet', {'mu': 6.}), 'F64'),
    (40000, 2, ('gmw', {'gamma': 3., 'beta': 60.}), 'F32'),
]


@pytest.fixture(scope='module')
def cuda():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return L.load()


def _run(lib, c, ex):
    code = getattr(L, c['prec'])
    args0 = (L.ptr(c['x']), c['B'], c['N'], c['Npad'], c['n1'], 1, 0, L.ptr(c['sc']))
    args1 = (c['na'], c['cw'], 1.0, c['cb'], c['gamma'], code, L.ptr(c['Wx']), None, None,
             L.ptr(c['idx']), c['ip'], L.ptr(c['ws']), c['wsb'], L.stream_ptr())
    c['Wx'].fill_(float('nan'))
    c['idx'].fill_(0x7777)
    if ex:
        rc = lib.ssqb_cwt_ex(*args0, c['sc_h'].ctypes.data, *args1)
    else:
        rc = lib.ssqb_cwt(*args0, *args1)
    L.check(rc, 'cwt')
    torch.cuda.synchronize()
    return c['Wx'].cpu().numpy(), c['idx'].cpu().numpy()[..., :c['N']]


@pytest.mark.parametrize('N, B, wav, prec', CASES)
def test_band_path_equals_tile_passes(cuda, N, B, wav, prec):
    f64 = prec == 'F64'
    w = P.Wavelet((wav[0], dict(wav[1], dtype='float64')))
    sc, st, na, nv = P.process_scales('log-piecewise', N, w, nv=32, get_params=True)
    f = P.compute_associated_frequencies(sc, N, w, st, 'peak', True, 1., 'cwt')
    mode, bp = P.bin_params(f, True)
    Npad, n1, _ = P.p2up(N)
    dev = torch.device('cuda', 0)
    xs = np.stack([S.chirp_mix(N, np.random.default_rng(50 + b)) for b in range(B)])
    ip = L.idx_pitch(N)
    code = getattr(L, prec)
    wsb = cuda.ssqb_cwt_workspace_bytes(B, N, Npad, na, code)
    c = dict(N=N, B=B, na=na, Npad=Npad, n1=n1, prec=prec, ip=ip, wsb=wsb,
             x=torch.as_tensor(xs.astype(np.float64 if f64 else np.float32), device=dev),
             sc=torch.as_tensor(sc.ravel(), dtype=torch.float64, device=dev),
             sc_h=np.ascontiguousarray(sc.ravel(), np.float64),
             cw=L.wavelet_struct(w), cb=L.make_bins(mode, bp, na, True),
             gamma=10 * (P.EPS64 if f64 else P.EPS32),
             Wx=torch.empty((B, na, N), dtype=torch.complex128 if f64 else torch.complex64,
                            device=dev),
             idx=torch.empty((B, na, ip), dtype=torch.uint16, device=dev),
             ws=torch.empty(wsb, dtype=torch.uint8, device=dev))
    W0, k0 = _run(cuda, c, ex=False)
    W1, k1 = _run(cuda, c, ex=True)
    assert np.isfinite(W1).all() and (k1 != 0x7777).all()
    e = rel_l2(W1, W0)
    flips = int((k1 != k0).sum())
    print(f'\nband path N={N} B={B} {wav[0]} {prec}: Wx rel-L2 {e:.2e}, bin differences '
          f'{flips} of {k0.size}')
    assert e <= {'F64': 1e-13, 'F32X': 1e-7, 'F32': 1e-5}[prec]
    assert flips <= (2 if prec != 'F32' else 1e-3 * k0.size)  # exact ties only
    assert L.device_status() == 0
