# -*- coding: utf-8 -*-
"""Reverse-mode differentiation: the adjoint kernels behind `cwt`, `ssq_cwt`,
`icwt`, `stft` and `ssq_stft` (ssqb_cwt_adjoint, ssqb_stft_adjoint,
ssqb_squeeze_adjoint, ssqb_icwt_adjoint).

CPU: argument checks of the adjoint entry points (no device call).
GPU: each adjoint against the float64 oracle's transposes (which the CPU
suite pins by the dot-product identity); the gradient of the batch-training
loss MSE(|Tx(x)|, |Tx(y)|) + MSE(icwt(Wx(x)), y) against float64 central
finite differences (eps = 1e-6, 32 random coordinates, bins held fixed) and
against a torch.fft composite of the same loss differentiated by torch's
own autograd in float64."""
import ctypes

import numpy as np
import pytest

from ssqueezepy_b200 import _lib as L
from ssqueezepy_b200 import _params as P
from ssqueezepy_b200 import _signals as S


def _adj(**kw):
    lib = L.load()
    p = ctypes.c_void_p(8)
    a = dict(gW=p, gT=None, idx=None, ip=0, sqw=None, nb=0, gx_r=None, icw=None, B=1,
             N=100, Npad=256, n1=78, pad=1, sc=p, na=10,
             wav=L.make_wavelet(0, (6., 1e-8, 1., 0.)), prec=L.F32, gx=p, acc=0, ws=p,
             wsb=1 << 30)
    a.update(kw)
    return lib.ssqb_cwt_adjoint(a['gW'], a['gT'], a['idx'], a['ip'], a['sqw'], a['nb'],
                                a['gx_r'], a['icw'], a['B'], a['N'], a['Npad'], a['n1'],
                                a['pad'], a['sc'], a['na'], a['wav'], a['prec'], a['gx'],
                                a['acc'], a['ws'], a['wsb'], None)


@pytest.mark.parametrize('kw, code', [
    (dict(gW=None), L.EINVAL),                                  # no source
    (dict(gT=ctypes.c_void_p(8)), L.EINVAL),                    # gTx without idx
    (dict(gT=ctypes.c_void_p(8), idx=ctypes.c_void_p(8), sqw=ctypes.c_void_p(8),
          nb=10, ip=50), L.EINVAL),                             # idx pitch < N
    (dict(gx_r=ctypes.c_void_p(8)), L.EINVAL),                  # icwt source w/o weights
    (dict(pad=3), L.EUNSUPPORTED),                              # replicate
    (dict(Npad=300), L.EUNSUPPORTED),
    (dict(n1=200), L.EINVAL),
    (dict(prec=5), L.EINVAL),
    (dict(wsb=64), L.EWORKSPACE),
    (dict(gx=None), L.EINVAL),
])
def test_cwt_adjoint_rejects_bad_arguments(kw, code):
    assert _adj(**kw) == code
    assert L.load().ssqb_last_error()


def test_wx_adjoints_reject_bad_arguments():
    lib = L.load()
    p = ctypes.c_void_p(8)
    assert lib.ssqb_squeeze_adjoint(None, p, 0, p, 1, 10, 10, 10, 0, p, 0, None) == L.EINVAL
    assert lib.ssqb_squeeze_adjoint(p, None, 0, p, 1, 10, 10, 10, 0, p, 0, None) == L.EINVAL
    assert lib.ssqb_squeeze_adjoint(p, p, 0, p, 1, 10, 10, 0, 0, p, 0, None) == L.EINVAL
    assert lib.ssqb_icwt_adjoint(p, None, 1, 10, 10, 0, p, 0, None) == L.EINVAL
    assert lib.ssqb_icwt_adjoint(p, p, 0, 10, 10, 0, p, 0, None) == L.EINVAL
    ws1 = lib.ssqb_cwt_adjoint_workspace_bytes(4, 1 << 15, 300, L.F32)
    ws2 = lib.ssqb_cwt_adjoint_workspace_bytes(4, 1 << 15, 300, L.F64)
    assert ws2 > ws1 > 4 * (1 << 15) * 12
    assert lib.ssqb_cwt_adjoint_workspace_bytes(0, 1 << 15, 300, L.F32) == 0


#### GPU ######################################################################
def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


MORLET = ('morlet', {'mu': 6.})


def _scales(N, dtype='float32'):
    w = P.Wavelet(('morlet', {'mu': 6., 'dtype': dtype}))
    return P.process_scales('log-piecewise', N, w, nv=32).ravel()


@pytest.mark.gpu
@pytest.mark.parametrize('N', [2000, 5000])      # Npad 4096 (one pass), 8192 (two)
@pytest.mark.parametrize('dtype', ['float32', 'float64'])
@pytest.mark.parametrize('padtype', ['reflect', 'zero'])
def test_cwt_backward_matches_oracle_adjoint(N, dtype, padtype):
    torch = _torch()
    import ssqueezepy_b200 as sb
    from oracle import ssq_oracle as O
    rng = np.random.default_rng(N)
    x = torch.tensor(S.same_length_batch(2, N, 1), device='cuda',
                     dtype=getattr(torch, dtype), requires_grad=True)
    Wx, sc = sb.cwt(x, ('morlet', {'mu': 6., 'dtype': dtype}), padtype=padtype)
    g = rng.standard_normal(Wx.shape) + 1j * rng.standard_normal(Wx.shape)
    (gx,) = torch.autograd.grad(Wx, x, torch.as_tensor(g, dtype=Wx.dtype, device='cuda'))
    ref = O.cwt_adjoint(g, 'morlet', (6.,), _scales(N, dtype), padtype=padtype)
    err = np.linalg.norm(gx.double().cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= (1e-5 if dtype == 'float32' else 1e-11), err
    assert L.device_status() == 0


@pytest.mark.gpu
def test_ssq_cwt_backward_is_gather_then_transpose():
    """dL/dx through (Tx, Wx) = cwt_adjoint(gWx + squeeze_adjoint(gTx)) with
    the forward's bins."""
    torch = _torch()
    import ssqueezepy_b200 as sb
    from oracle import ssq_oracle as O
    from ssqueezepy_b200 import _transforms as T
    N = 6000
    x = torch.tensor(S.same_length_batch(1, N, 2)[0], device='cuda', dtype=torch.float32,
                     requires_grad=True)
    Tx, Wx, f, sc = sb.ssq_cwt(x, MORLET)
    rng = np.random.default_rng(1)
    gT = rng.standard_normal(Tx.shape) + 1j * rng.standard_normal(Tx.shape)
    gW = rng.standard_normal(Wx.shape) + 1j * rng.standard_normal(Wx.shape)
    (gx,) = torch.autograd.grad((Tx, Wx), x,
                                (torch.as_tensor(gT, dtype=Tx.dtype, device='cuda'),
                                 torch.as_tensor(gW, dtype=Wx.dtype, device='cuda')))
    # bins of the forward, from the plain call's bin index
    wav = P.Wavelet(('morlet', {'mu': 6.}))
    r = T._cwt_core(x.detach(), wav, 'log-piecewise', 32, None, None, 'reflect', False,
                    False, False, want_idx=True,
                    ssq=(*P.bin_params(f[::-1].copy(), True), len(f), True))
    k = r['idx'][0, :, :N].cpu().numpy().astype(np.int64)
    use = k != L.NO_BIN
    k = np.where(use, k, 0)
    fp = T._ssq_plan(wav, 'log-piecewise', N, 32, None, 'peak', 'reflect', 1.)
    gWtot = gW + O.squeeze_adjoint(gT, k, use, fp['const'])
    ref = O.cwt_adjoint(gWtot, 'morlet', (6.,), _scales(N))
    err = np.linalg.norm(gx.double().cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= 1e-5, err


@pytest.mark.gpu
def test_icwt_backward_is_row_weights_times_gradient():
    torch = _torch()
    import ssqueezepy_b200 as sb
    from ssqueezepy_b200 import _transforms as T
    N, na = 4000, len(_scales(4000))
    rng = np.random.default_rng(3)
    W = torch.tensor(rng.standard_normal((2, na, N)) + 1j * rng.standard_normal((2, na, N)),
                     dtype=torch.complex64, device='cuda', requires_grad=True)
    xr = sb.icwt(W, ('morlet', {'mu': 6.}), x_len=N)
    g = torch.randn_like(xr)
    (gW,) = torch.autograd.grad(xr, W, g)
    wav = P.process_gmw_wavelet(('morlet', {'mu': 6.}), True)
    wts = T._icwt_plan(P.Wavelet._init_if_not_isinstance(wav), 'log-piecewise', N, 32,
                       True)['weights']
    ref = wts[None, :, None] * g.double().cpu().numpy()[:, None, :]
    got = gW.cpu().numpy()
    assert np.abs(got.imag).max() == 0
    assert np.linalg.norm(got.real - ref) <= 1e-6 * np.linalg.norm(ref)


def _loss_parts(sb, torch, x, y, Ty_abs):
    Tx, Wx, f, sc = sb.ssq_cwt(x, MORLET)
    xr = sb.icwt(Wx, ('morlet', {'mu': 6.}), x_len=x.shape[-1])
    return ((Tx.abs() - Ty_abs) ** 2).mean() + ((xr - y) ** 2).mean(), Tx, Wx, f, sc


@pytest.mark.gpu
@pytest.mark.parametrize('B, N, comp', [(4, 4096, 4), (64, 16384, 4)])
def test_training_loss_gradient_vs_finite_differences_and_torch_composite(B, N, comp):
    """Loss = MSE(|Tx(x)|, |Tx(y)|) + MSE(icwt(Wx(x)), y) on a batch of B
    signals of length N from the chirp-mixture family: 4 x 4096, and the
    differentiable-training workload itself, 64 x 16,384 (padded 32,768,
    301 rows). The finite differences take 32 coordinates over all signals;
    the torch composite runs on the first `comp` signals (the loss is a sum
    of per-signal terms, so those rows of the gradient are the full batch's)."""
    torch = _torch()
    import ssqueezepy_b200 as sb
    from oracle import ssq_oracle as O
    from ssqueezepy_b200 import _transforms as T
    xs = S.same_length_batch(B, N, 5678)
    ys = S.same_length_batch(B, N, 9012)
    y = torch.tensor(ys, dtype=torch.float32, device='cuda')
    with torch.no_grad():
        Ty = sb.ssq_cwt(y, MORLET)[0]
    x = torch.tensor(xs, dtype=torch.float32, device='cuda', requires_grad=True)
    loss, Tx, Wx, f, sc = _loss_parts(sb, torch, x, y, Ty.abs())
    loss.backward()
    g_ours = x.grad.double().cpu().numpy()

    # fixed bins of the forward (the gradient treats them as constants)
    wav = P.Wavelet(('morlet', {'mu': 6.}))
    r = T._cwt_core(x.detach(), wav, 'log-piecewise', 32, None, None, 'reflect', False,
                    False, False, want_idx=True,
                    ssq=(*P.bin_params(f[::-1].copy(), True), len(f), True))
    k = r['idx'][..., :N].cpu().numpy().astype(np.int64)
    use = k != L.NO_BIN
    k = np.where(use, k, 0)
    fp = T._ssq_plan(wav, 'log-piecewise', N, 32, None, 'peak', 'reflect', 1.)
    const = fp['const']
    ip = T._icwt_plan(wav, 'log-piecewise', N, 32, True)
    wts, mm = ip['weights'], ip['mean_mult']
    s64 = _scales(N)
    Tya = Ty.abs().double().cpu().numpy()
    na = len(s64)

    def loss_np(xb, b):  # float64 loss term of signal b, bins fixed
        Wb, _ = O.cwt(xb, 'morlet', (6.,), s64, derivative=False)
        Tb = O.squeeze(Wb, k[b], use[b], const)
        xr = (wts[:, None] * Wb.real).sum(0)
        return (((np.abs(Tb) - Tya[b]) ** 2).sum() / (B * na * N)
                + ((xr - ys[b]) ** 2).sum() / (B * N))

    x32 = xs.astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(0)
    coords = [(int(rng.integers(B)), int(rng.integers(N))) for _ in range(32)]
    eps = 1e-6
    fd = []
    for b, j in coords:
        xp, xm = x32[b].copy(), x32[b].copy()
        xp[j] += eps
        xm[j] -= eps
        fd.append((loss_np(xp, b) - loss_np(xm, b)) / (2 * eps))
    fd = np.array(fd)
    ours = np.array([g_ours[b, j] for b, j in coords])
    e_fd = np.linalg.norm(ours - fd) / np.linalg.norm(fd)
    assert e_fd <= 1e-3, e_fd

    # torch.fft composite in float64 on the CPU, same fixed bins, signals
    # [0, comp) with the full batch's normalisation
    xt = torch.tensor(x32[:comp], dtype=torch.float64, requires_grad=True)
    k, use, Tya, ys_c = k[:comp], use[:comp], Tya[:comp], ys[:comp]
    Npad, n1, n2 = P.p2up(N)
    src = torch.as_tensor(O.pad_sources(N, 'reflect', n1, n2))
    Ph = torch.as_tensor(O.psih_bank('morlet', (6.,), s64, Npad)[0])
    Wt = torch.fft.ifft(Ph * torch.fft.fft(xt[:, src], dim=-1)[:, None, :],
                        dim=-1)[..., n1:n1 + N]
    V = Wt * (torch.as_tensor(const)[None, :, None] * torch.as_tensor(use, dtype=torch.float64))
    kt = torch.as_tensor(k)
    z = torch.zeros(Wt.shape, dtype=torch.float64)
    Tt = torch.complex(z.scatter_add(1, kt, V.real), z.scatter_add(1, kt, V.imag))
    xr = (torch.as_tensor(wts)[None, :, None] * Wt.real).sum(1) + 0 * mm
    lt = (((Tt.abs() - torch.as_tensor(Tya)) ** 2).sum() / (B * na * N)
          + ((xr - torch.as_tensor(ys_c)) ** 2).sum() / (B * N))
    lt.backward()
    g_ref = xt.grad.numpy()
    e_tc = np.linalg.norm(g_ours[:comp] - g_ref) / np.linalg.norm(g_ref)
    print(f'\nB={B} N={N}: gradient vs FD {e_fd:.2e}, vs torch composite {e_tc:.2e}')
    assert e_tc <= 1e-4, e_tc
    if comp == B:
        assert abs(float(loss) - float(lt)) <= 1e-4 * abs(float(lt))


@pytest.mark.gpu
@pytest.mark.parametrize('dtype', ['float32', 'float64'])
@pytest.mark.parametrize('hop, padtype', [(1, 'reflect'), (2, 'zero'), (3, 'reflect')])
def test_stft_backward_matches_oracle_adjoint(dtype, hop, padtype):
    torch = _torch()
    import ssqueezepy_b200 as sb
    from oracle import ssq_oracle as O
    from scipy.signal import get_window
    N, n_fft = 3000, 256
    rng = np.random.default_rng(hop)
    x = torch.tensor(S.same_length_batch(2, N, 3), device='cuda',
                     dtype=getattr(torch, dtype), requires_grad=True)
    Sx = sb.stft(x, window='hann', n_fft=n_fft, hop_len=hop, padtype=padtype, dtype=dtype)
    g = rng.standard_normal(Sx.shape) + 1j * rng.standard_normal(Sx.shape)
    (gx,) = torch.autograd.grad(Sx, x, torch.as_tensor(g, dtype=Sx.dtype, device='cuda'))
    win = get_window('hann', n_fft, fftbins=True)
    ref = O.stft_adjoint(g, win, n_fft, N, hop=hop, padtype=padtype)
    err = np.linalg.norm(gx.double().cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= (1e-5 if dtype == 'float32' else 1e-11), err
    assert L.device_status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize('dtype', ['float32', 'float64'])
@pytest.mark.parametrize('n_fft, hop', [(121, 1), (100, 2), (598, 3)])
def test_stft_backward_any_length_matches_oracle_adjoint(dtype, n_fft, hop):
    """n_fft not a power of two: the frame transform of the backward goes
    through the chirp-z kernel, the gather rotates modulo n_fft."""
    torch = _torch()
    import ssqueezepy_b200 as sb
    from oracle import ssq_oracle as O
    from scipy.signal import get_window
    N = 1500
    rng = np.random.default_rng(n_fft)
    x = torch.tensor(S.same_length_batch(2, N, 5), device='cuda',
                     dtype=getattr(torch, dtype), requires_grad=True)
    Sx = sb.stft(x, window='hann', n_fft=n_fft, hop_len=hop, dtype=dtype)
    g = rng.standard_normal(Sx.shape) + 1j * rng.standard_normal(Sx.shape)
    (gx,) = torch.autograd.grad(Sx, x, torch.as_tensor(g, dtype=Sx.dtype, device='cuda'))
    win = get_window('hann', n_fft, fftbins=True)
    ref = O.stft_adjoint(g, win, n_fft, N, hop=hop)
    err = np.linalg.norm(gx.double().cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= (1e-5 if dtype == 'float32' else 1e-11), err
    assert L.device_status() == 0


@pytest.mark.gpu
def test_ssq_stft_backward_is_gather_then_transpose():
    torch = _torch()
    import ssqueezepy_b200 as sb
    from oracle import ssq_oracle as O
    from scipy.signal import get_window
    from ssqueezepy_b200 import _transforms as T
    N, n_fft = 4000, 128
    x = torch.tensor(S.same_length_batch(1, N, 4)[0], device='cuda', dtype=torch.float32,
                     requires_grad=True)
    Tx, Sx, f, Sfs = sb.ssq_stft(x, window='hann', n_fft=n_fft)
    rng = np.random.default_rng(2)
    gT = rng.standard_normal(Tx.shape) + 1j * rng.standard_normal(Tx.shape)
    gS = rng.standard_normal(Sx.shape) + 1j * rng.standard_normal(Sx.shape)
    (gx,) = torch.autograd.grad((Tx, Sx), x,
                                (torch.as_tensor(gT, dtype=Tx.dtype, device='cuda'),
                                 torch.as_tensor(gS, dtype=Sx.dtype, device='cuda')))
    nrow = n_fft // 2 + 1
    Sfs64 = np.linspace(0, .5, nrow)
    mode, bp = P.bin_params(Sfs64, False)
    r = T._stft_core(x.detach(), 'hann', n_fft, None, 1, None, None, 'reflect', True, False,
                     'float32', want_idx=True, bins=(mode, bp))
    k = r['idx'][0, :, :N].cpu().numpy().astype(np.int64)
    use = k != L.NO_BIN
    k = np.where(use, k, 0)
    gStot = gS + O.squeeze_adjoint(gT, k, use, Sfs64[1] - Sfs64[0])
    ref = O.stft_adjoint(gStot, get_window('hann', n_fft, fftbins=True), n_fft, N)
    err = np.linalg.norm(gx.double().cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= 1e-5, err
