# -*- coding: utf-8 -*-
"""The long-signal workload against the float64 oracle: one float32 chirp
mixture of N = 1,048,576 samples (padded 2,097,152, the largest two-pass
transform), GMW gamma=3 beta=60, scales='log:maximal' (613 rows).

Checked: the norm of every Wx row, eight whole rows, and Tx and the bin
index over a window of columns (Tx of a column needs every row of it, so
the oracle squeezes the window's columns of all rows). The oracle is
computed in chunks of rows to bound its memory."""
import numpy as np
import pytest
import torch

from oracle import ssq_oracle as O
from ssqueezepy_b200 import _params as P
from ssqueezepy_b200 import _signals as S
from ssqueezepy_b200 import _transforms as T
from tests._cases import rel_l2

pytestmark = pytest.mark.gpu

N = 1 << 20
GMW = ('gmw', {'gamma': 3., 'beta': 60., 'dtype': 'float32'})


@pytest.fixture(scope='module')
def sb():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as m
    m._lib.load()
    return m


def _oracle_rows(x64, s64, rows, c0, C, chunk=24):
    """Row norms of Wx, the window [c0, c0 + C) of Wx and dWx for every row,
    and the whole rows `rows`."""
    Npad, n1, n2 = O.p2up(len(x64))
    xh = np.fft.fft(O.pad(x64, 'reflect', n1, n2))
    norms = np.empty(len(s64))
    Wwin = np.empty((len(s64), C), np.complex128)
    dWwin = np.empty_like(Wwin)
    full = {}
    for i0 in range(0, len(s64), chunk):
        sl = slice(i0, min(i0 + chunk, len(s64)))
        Pb, xi = O.psih_bank('gmw_l1', (3., 60.), s64[sl], Npad)
        Z = Pb * xh
        W = O.sfft.ifft(Z, axis=-1, workers=O._WORKERS)[:, n1:n1 + len(x64)]
        Z *= 1j * xi
        dW = O.sfft.ifft(Z, axis=-1, workers=O._WORKERS)[:, n1:n1 + len(x64)]
        norms[sl] = np.linalg.norm(W, axis=1)
        Wwin[sl] = W[:, c0:c0 + C]
        dWwin[sl] = dW[:, c0:c0 + C]
        for i in rows:
            if sl.start <= i < sl.stop:
                full[i] = W[i - sl.start].copy()
    return norms, Wwin, dWwin, full


def test_long_signal_vs_oracle(sb):
    x32 = S.chirp_mix(N, np.random.default_rng(4321)).astype(np.float32)
    wav = P.Wavelet(GMW)
    fp = T._ssq_plan(wav, 'log:maximal', N, 32, None, 'peak', 'reflect', 1.)
    sp = T._scales_plan('log:maximal', N, wav, 32)
    s64, na = sp['scales'], sp['na']
    assert na == 613
    xd = torch.as_tensor(x32, device='cuda')
    Tx, Wx, f, sc = sb.ssq_cwt(xd, GMW, scales='log:maximal')
    r = T._cwt_core(xd, wav, 'log:maximal', 32, None, None, 'reflect', False, False,
                    False, want_idx=True, ssq=(fp['mode'], fp['bp'], na, True))
    c0, C = 300000, 8192
    rows = [0, 100, 250, 400, 500, 560, 600, 612]
    norms_g = torch.linalg.vector_norm(Wx, dim=-1).double().cpu().numpy().ravel()
    Wwin_g = Wx[..., c0:c0 + C].cpu().numpy().reshape(na, C)
    Twin_g = Tx[..., c0:c0 + C].cpu().numpy().reshape(na, C)
    idx_g = r['idx'][0, :, c0:c0 + C].cpu().numpy()
    full_g = {i: Wx[..., i, :].cpu().numpy().ravel() for i in rows}
    del Tx, Wx, r
    torch.cuda.empty_cache()

    norms, Wwin, dWwin, full = _oracle_rows(x32.astype(np.float64), s64, rows, c0, C)
    e_norm = np.max(np.abs(norms_g - norms) / norms.max())
    e_rows = max(rel_l2(full_g[i], full[i]) for i in rows)
    e_win = rel_l2(Wwin_g, Wwin)
    gamma = 10 * P.EPS32
    rep = O.bin_parity(idx_g, Wwin, dWwin, fp['f_asc'], fp['mode'] != 2, True, gamma)
    w = O.phase_cwt(Wwin, dWwin, gamma)
    use = np.abs(Wwin) > gamma
    k = O.bin_index(np.where(use, w, 1.), fp['f_asc'], fp['mode'] != 2, True)
    Twin = O.squeeze(Wwin, k, use, fp['const'])
    e_tx = rel_l2(Twin_g, Twin)
    print(f'\nN=2^20 613 rows: row norms {e_norm:.2e}, rows {e_rows:.2e}, '
          f'window Wx {e_win:.2e}, window Tx {e_tx:.2e}, bins {rep}')
    assert e_norm <= 1e-6
    assert e_rows <= 1e-5 and e_win <= 1e-5
    assert e_tx <= 1e-4
    assert rep['other'] == 0 and rep['mask_other'] == 0, rep
