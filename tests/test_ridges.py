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


def _ridge_field(nf, N, dtype, seed=0):
    """Two drifting ridges over complex noise, nf rows x N columns."""
    rng = np.random.default_rng(seed)
    f = np.arange(nf)[:, None]
    t = np.arange(N)[None, :]
    c1 = nf * (0.3 + 0.2 * np.sin(2 * np.pi * t / N))
    c2 = nf * (0.7 - 0.1 * t / N)
    amp = (np.exp(-0.5 * ((f - c1) / (0.01 * nf + 1)) ** 2)
           + 0.7 * np.exp(-0.5 * ((f - c2) / (0.01 * nf + 1)) ** 2))
    noise = 0.05 * (rng.standard_normal((nf, N)) + 1j * rng.standard_normal((nf, N)))
    return (amp + noise).astype(dtype)


def _gpu_track_on_own_E(T, sc, penalty=2.):
    """One ridge through the C ABI, then the oracle's sweep over the E the
    GPU computed (read back from the workspace: energy, E, pen, each (N, nf)
    time-major for E and pen): the sweeps' indices without the log's
    rounding."""
    import torch
    from oracle import ssq_oracle as O
    nf, N = T.shape
    dt = np.float32
    Td = torch.as_tensor(T, device='cuda')
    s = np.log(sc.astype(dt))
    s_d = torch.as_tensor(s, device='cuda')
    sc_d = torch.as_tensor(sc.astype(dt), device='cuda')
    idx = torch.empty((N, 1), dtype=torch.int32, device='cuda')
    lib = L.load()
    wsb = lib.ssqb_ridges_workspace_bytes(nf, N, L.F32)
    ws = torch.zeros(wsb, dtype=torch.uint8, device='cuda')
    rc = lib.ssqb_extract_ridges(L.ptr(Td), nf, N, L.ptr(s_d), L.ptr(sc_d), float(penalty), 1,
                                 4, float(np.finfo(dt).eps), L.F32, L.ptr(idx), None, None,
                                 L.ptr(ws), wsb, L.stream_ptr())
    L.check(rc, 'extract_ridges')
    n = nf * N
    E = ws[:4 * 2 * n].view(torch.float32)[n:2 * n].view(N, nf).T.cpu().numpy()
    P = dt(penalty) * np.subtract.outer(s, s) ** 2
    return idx[:, 0].cpu().numpy(), O.ridge_track(E.copy(), P, dt(np.finfo(dt).eps))


@pytest.mark.gpu
@pytest.mark.parametrize('nf', [40, 300, 600, 1200, 9000])
@pytest.mark.parametrize('dtype', [np.complex64, np.complex128])
def test_ridges_match_oracle_across_sweep_variants(nf, dtype):
    """Row counts that select each forward variant (cluster with register
    penalties, cluster with computed penalties at 8 and 4 lanes per row,
    single-CTA) and each backward variant (staged warp with 4 / 10 / 32 rows
    per lane, block-wide), against the oracle: indices bit-exact. For float32
    at 9000 rows (ridges 90 rows wide, so paths whose costs part by less than
    an ulp of E) the sweeps are checked on the GPU's own E: numpy's float32
    log is a SIMD approximation, not correctly rounded, and it and CUDA's
    part by an ulp on many inputs, which the re-tracking's exact-equality
    test can turn into a different row."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ssqueezepy_b200 as sb
    from oracle import ssq_oracle as O
    N = 120 if nf < 9000 else 6
    T = _ridge_field(nf, N, dtype, seed=nf)
    sc = np.geomspace(1., 300., nf)
    if nf == 9000 and dtype == np.complex64:
        got, want = _gpu_track_on_own_E(T, sc)
        assert np.array_equal(got, want)
        assert L.device_status() == 0
        return
    i, f, e = sb.extract_ridges(T, sc, penalty=2., n_ridges=2, bw=max(2, nf // 40),
                                get_params=True)
    io, fo, eo = O.extract_ridges(T, sc, penalty=2., n_ridges=2, bw=max(2, nf // 40))
    assert L.device_status() == 0
    assert np.array_equal(i, io)
    assert np.array_equal(f, fo)
    assert np.allclose(e, eo, rtol=1e-6 if dtype == np.complex64 else 1e-13)
