# -*- coding: utf-8 -*-
"""CPU float64 restatement of ssqueezepy's synchrosqueezing hot path.

TEST INFRASTRUCTURE ONLY. This module is the checker: only `tests/`,
`__graft_entry__.smoke()` and the CPU-baseline / reference arm of `bench.py`
may import it. The product (`ssqueezepy_b200`) never calls it and has no CPU
fallback.

Each function restates the reference routine it cites (paths relative to the
ssqueezepy source tree) in plain numpy / scipy.fft, float64 throughout, the
way ssqueezepy computes with a float64 `Wavelet`. It is pinned against
outputs of ssqueezepy itself: tests/golden/*.npz, generated by
tests/golden/make_golden.py (see tests/test_oracle.py).

Host parameters (scales, ssq_freqs, per-row weights) are inputs here; they
are pinned separately against the same fixtures (tests/test_params.py).
"""
import os
import numpy as np
from concurrent.futures import ThreadPoolExecutor
from scipy import fft as sfft

PI = np.pi
EPS32 = float(np.finfo(np.float32).eps)
EPS64 = float(np.finfo(np.float64).eps)
_WORKERS = os.cpu_count() or 1


#### padding (utils/common.py:32-51, 54-158) ##################################
def p2up(n):
    up = int(2 ** (1 + np.round(np.log2(n))))
    n2 = (up - n) // 2
    return up, up - n - n2, n2


def pad(x, padtype, n1, n2):
    """Pad the last axis by (n1, n2) with numpy's modes, as padsignal does."""
    widths = [(0, 0)] * (x.ndim - 1) + [(n1, n2)]
    if padtype == 'zero':
        return np.pad(x, widths)
    if padtype == 'reflect':
        return np.pad(x, widths, mode='reflect')
    if padtype == 'replicate':
        return np.pad(x, widths, mode='edge')
    if padtype == 'wrap':
        return np.pad(x, widths, mode='wrap')
    if padtype == 'symmetric':
        r = x[..., ::-1]
        return np.concatenate([r[..., r.shape[-1] - n1:], x, r[..., :n2]], -1)
    raise ValueError(padtype)


#### wavelets (wavelets.py:473-530, _gmw.py:187-251) ##########################
def xi_grid(N):
    """[0, .., N//2, -(N-N//2-1), .., -1] * 2pi/N (wavelets.py:473-484)."""
    h = 2 * PI / N
    k = np.arange(N, dtype=np.float64)
    k[N // 2 + 1:] -= N
    return k * h


def psih(kind, params, w):
    """Frequency-domain wavelet at radian frequencies `w`.

    kind 'morlet': params (mu,): C1*(exp(-(w-mu)^2/2) - ks*exp(-w^2/2)),
      ks = exp(-mu^2/2), C1 = sqrt(2)*cs*pi^(1/4),
      cs = (1 + exp(-mu^2) - 2exp(-3mu^2/4))^(-1/2)   (wavelets.py:498-527)
    kind 'gmw_l1': params (gamma, beta): 2exp(-beta ln wc + wc^gamma
      + beta ln w - w^gamma) for w >= 0, wc = (beta/gamma)^(1/gamma)
                                                     (_gmw.py:187-210, 638)
    kind 'gmw_l2': params (gamma, beta): sqrt(2pi gamma 2^r / Gamma(r))
      w^beta exp(-w^gamma), r = (2beta+1)/gamma      (_gmw.py:228-251)
    GMW params (gamma, beta, k), k > 0: the order-k wavelet, the order-0
      exponential times the generalized Laguerre polynomial L_k^c(2w^gamma),
      c = r - 1, and the order-k norm: 2 sqrt(Gamma(r) k! / Gamma(k+r)) for
      'gmw_l1', sqrt(2pi gamma 2^r k! / Gamma(k+r)) for 'gmw_l2'
                                       (_gmw.py:268-296, 320-347, 368-396)
    """
    w = np.asarray(w, dtype=np.float64)
    if kind == 'morlet':
        mu, = params
        cs = (1 + np.exp(-mu**2) - 2 * np.exp(-3 / 4 * mu**2)) ** (-.5)
        ks = np.exp(-.5 * mu**2)
        C1 = np.sqrt(2) * cs * PI**.25
        return C1 * (np.exp(-.5 * (w - mu)**2) - ks * np.exp(-.5 * w**2))
    gamma, beta = params[:2]
    k = int(params[2]) if len(params) > 2 else 0
    wc = (beta / gamma) ** (1 / gamma)
    nonneg = w >= 0
    w = w * nonneg
    if k > 0:
        from scipy.special import eval_genlaguerre, gammaln
        r = (2 * beta + 1) / gamma
        lag = eval_genlaguerre(k, r - 1, 2 * w**gamma)
        with np.errstate(divide='ignore'):
            if kind == 'gmw_l1':
                norm = 2 * np.sqrt(np.exp(gammaln(r) + gammaln(k + 1) - gammaln(k + r)))
                base = np.exp(-beta * np.log(wc) + wc**gamma + beta * np.log(w) - w**gamma)
            else:
                norm = np.sqrt(2 * PI * gamma * 2.**r
                               * np.exp(gammaln(k + 1) - gammaln(k + r)))
                base = np.exp(beta * np.log(w) - w**gamma)
        return norm * lag * base * nonneg
    with np.errstate(divide='ignore'):
        if kind == 'gmw_l1':
            return 2 * np.exp(-beta * np.log(wc) + wc**gamma
                              + beta * np.log(w) - w**gamma) * nonneg
        from scipy.special import gamma as gamma_fn
        r = (2 * beta + 1) / gamma
        return (np.sqrt(2. * PI * gamma * 2.**r / gamma_fn(r))
                * w**beta * np.exp(-w**gamma) * nonneg)
    raise ValueError(kind)


def psih_bank(kind, params, scales, Npad):
    """psih(scale * xi) for every scale, Nyquist bin halved for even Npad
    (wavelets.py:62-95, _cwt.py:167-171 with nohalf=False)."""
    xi = xi_grid(Npad)
    P = psih(kind, params, np.asarray(scales, np.float64).reshape(-1, 1) * xi)
    if Npad % 2 == 0:
        P[:, Npad // 2] /= 2
    return P, xi


#### CWT (_cwt.py:167-177, 246-320) ###########################################
def cwt(x, kind, params, scales, dt=1., padtype='reflect', l1_norm=True,
        derivative=True):
    """Wx (and dWx) of 1D or 2D `x`, shape (..., na, N)."""
    x = np.asarray(x, dtype=np.float64)
    N = x.shape[-1]
    if padtype is None:
        Npad, n1 = N, 0
        xp = x
    else:
        Npad, n1, n2 = p2up(N)
        xp = pad(x, padtype, n1, n2)
    xh = sfft.fft(xp, axis=-1, workers=_WORKERS)
    P, xi = psih_bank(kind, params, scales, Npad)
    if x.ndim == 2:
        xh = xh[:, None]
    Pxh = P * xh
    Wx = sfft.ifft(Pxh, axis=-1, workers=_WORKERS)[..., n1:n1 + N]
    dWx = None
    if derivative:
        Pxh *= (1j * xi / dt)
        dWx = sfft.ifft(Pxh, axis=-1, workers=_WORKERS)[..., n1:n1 + N]
    if not l1_norm:
        s = np.sqrt(np.asarray(scales, np.float64).reshape(-1, 1))
        Wx = Wx * s
        if dWx is not None:
            dWx = dWx * s
    return np.ascontiguousarray(Wx), (None if dWx is None else
                                      np.ascontiguousarray(dWx))


def cwt_higher_order(x, kind, params, orders, scales, dt=1., padtype='reflect',
                     l1_norm=True, derivative=True):
    """Mean over `orders` of the order-k transforms, each `cwt` with the
    order-k GMW (cwt_higher_order, _cwt.py:586-599)."""
    outs = [cwt(x, kind, tuple(params[:2]) + (k,), scales, dt, padtype, l1_norm,
                derivative) for k in orders]
    Wx = np.mean([o[0] for o in outs], axis=0)
    dWx = np.mean([o[1] for o in outs], axis=0) if derivative else None
    return Wx, dWx


#### phase transform (algos.py:706-740, 784-816) ##############################
def phase_cwt(Wx, dWx, gamma):
    """|Im(dWx conj(Wx))| / (|Wx|^2 2pi); inf where |Wx| < gamma."""
    A, B = dWx.real, dWx.imag
    C, D = Wx.real, Wx.imag
    with np.errstate(divide='ignore', invalid='ignore'):
        w = np.abs((B * C - A * D) / ((C**2 + D**2) * 6.283185307179586))
    w[np.abs(Wx) < gamma] = np.inf
    return w


def phase_unwrap(Wx, gamma):
    """difftype='phase' (_ssq_cwt.py:490-496): steps of the angle of Wx
    unwrapped along time, the last column u[-1] - u[0]; |.| / 2pi, inf where
    |Wx| < gamma."""
    u = np.unwrap(np.angle(Wx), axis=-1)
    w = np.concatenate([np.diff(u, axis=-1), u[..., -1:] - u[..., :1]], axis=-1)
    w = np.abs(w / (2 * PI))
    w[np.abs(Wx) < gamma] = np.inf
    return w


def phase_numeric(Wx, dt, order, gamma):
    """phase_cwt_num (_ssq_cwt.py:512-586): periodic differences of order
    1, 2 or 4 along time, |Im(D Wx / Wx)| / 2pi, inf where |Wx| < gamma."""
    def sh(k):  # W[j + k], periodic
        return np.roll(Wx, -k, axis=-1)
    if order == 1:
        D = (sh(1) - Wx) / dt
    elif order == 2:
        D = (-sh(2) + 4 * sh(1) - 3 * Wx) / (2 * dt)
    else:
        D = (-sh(2) + 8 * sh(1) - 8 * sh(-1) + sh(-2)) / (12 * dt)
    w = np.abs(np.imag(D / Wx) / (2 * PI))
    w[np.abs(Wx) < gamma] = np.inf
    return w


def phase_stft(Sx, dSx, Sfs, gamma):
    """|Sfs_i - Im(dS conj(S)) / (|S|^2 2pi)|; inf where |S| < gamma."""
    A, B = dSx.real, dSx.imag
    C, D = Sx.real, Sx.imag
    Sfs = np.asarray(Sfs, np.float64).reshape(-1, 1)
    with np.errstate(divide='ignore', invalid='ignore'):
        w = np.abs(Sfs - (B * C - A * D) / ((C**2 + D**2) * 6.283185307179586))
    w[np.abs(Sx) < gamma] = np.inf
    return w


#### bins (algos.py:356-374, 859-984) #########################################
def transition_idx(v):
    """Split index of two log-spaced pieces, or None (cwt_utils.py:375-394)."""
    v = np.asarray(v)
    d2 = np.abs(np.diff(np.log(v), 2, axis=0)).ravel()
    idx = int(np.argmax(d2)) + 2
    mx = d2.max()
    d2[idx - 2] = 0
    th = 1e-14 if v.dtype == np.float64 else 1e-6
    if not np.any(mx > 100 * np.abs(d2).mean()):
        return None
    if not np.all(np.abs(d2) < th):
        return None
    return idx


def bin_index(w, ssq_freqs, logscale, flipud):
    """Frequency bin of each phase-transform value (round-half-even as numba's
    `round`); `w` must be finite where used."""
    v = np.asarray(ssq_freqs, np.float64).ravel()
    omax = len(v) - 1
    with np.errstate(divide='ignore', invalid='ignore'):
        if not logscale:
            dv = max(float(v[1] - v[0]), EPS64)
            k = np.minimum(np.round(np.maximum((w - v[0]) / dv, 0)), omax)
        else:
            idx = transition_idx(v)
            vlmin = float(np.log2(v[0]))
            wl = np.log2(w)
            if idx is None:
                dvl = max(float(np.log2(v[1]) - np.log2(v[0])), EPS64)
                k = np.minimum(np.round(np.maximum((wl - vlmin) / dvl, 0)), omax)
            else:
                vlmin1 = float(np.log2(v[idx - 1]))
                dvl0 = max(float(np.log2(v[1]) - np.log2(v[0])), EPS64)
                dvl1 = max(float(np.log2(v[idx]) - np.log2(v[idx - 1])), EPS64)
                hi = np.minimum(np.round((wl - vlmin1) / dvl1) + (idx - 1), omax)
                lo = np.maximum(np.round((wl - vlmin) / dvl0), 0)
                k = np.where(wl > vlmin1, hi, lo)
    k = np.where(np.isfinite(k), k, 0).astype(np.int64)
    if flipud:
        k = omax - k
    return k


def bin_edge_w(w, ssq_freqs, logscale):
    """Phase-transform value of the rounding edge nearest to each `w` under
    the bin rule of `bin_index` (algos.py:859-953), and of the split of a
    log-piecewise grid where that is nearer."""
    v = np.asarray(ssq_freqs, np.float64).ravel()
    with np.errstate(divide='ignore', invalid='ignore'):
        if not logscale:
            dv = max(float(v[1] - v[0]), EPS64)
            e = np.floor((w - v[0]) / dv) + .5
            return v[0] + e * dv
        wl = np.log2(w)
        idx = transition_idx(v)
        vlmin = float(np.log2(v[0]))
        if idx is None:
            dvl = max(float(np.log2(v[1]) - np.log2(v[0])), EPS64)
            return 2. ** (vlmin + (np.floor((wl - vlmin) / dvl) + .5) * dvl)
        vlmin1 = float(np.log2(v[idx - 1]))
        dvl0 = max(float(np.log2(v[1]) - np.log2(v[0])), EPS64)
        dvl1 = max(float(np.log2(v[idx]) - np.log2(v[idx - 1])), EPS64)
        hi = 2. ** (vlmin1 + (np.floor((wl - vlmin1) / dvl1) + .5) * dvl1)
        lo = 2. ** (vlmin + (np.floor((wl - vlmin) / dvl0) + .5) * dvl0)
        edge = np.where(wl > vlmin1, hi, lo)
        split = 2. ** vlmin1
        return np.where(np.abs(w - split) < np.abs(w - edge), split, edge)


def bin_parity(idx, Wx, dWx, ssq_freqs, logscale, flipud, gamma, no_bin=0xFFFF):
    """Compare a bin index computed elsewhere (`idx`, (na, N) integers,
    `no_bin` where |Wx| <= gamma) with the float64 bins of (Wx, dWx).

    Returns a dict of counts: entries, mismatched bins among entries both
    keep, of which `near_edge` have the float64 w within one float32 ulp of
    the rounding edge between the two bins (ties that float32 data cannot
    resolve), `other` the rest; mask disagreements, of which `near_gamma`
    have |Wx| within 1e-12 of gamma (relative)."""
    w = phase_cwt(Wx, dWx, gamma)
    a = np.abs(Wx)
    use = a > gamma
    k = bin_index(np.where(use, w, 1.), ssq_freqs, logscale, flipud)
    got = np.asarray(idx).astype(np.int64)
    keep = got != no_bin
    both = use & keep
    mis = both & (got != k)
    wm = w[mis]
    ulp = np.spacing(wm.astype(np.float32)).astype(np.float64)
    near = np.abs(wm - bin_edge_w(wm, ssq_freqs, logscale)) <= ulp
    mask_mis = use != keep
    near_g = np.abs(a[mask_mis] - gamma) <= 1e-12 * gamma
    return dict(entries=int(use.size), kept=int(use.sum()), mismatched=int(mis.sum()),
                near_edge=int(near.sum()), other=int((~near).sum()),
                mask_mismatched=int(mask_mis.sum()), mask_near_gamma=int(near_g.sum()),
                mask_other=int((~near_g).sum()))


def squeeze(Wx, k, use, const):
    """Tx[k[i,j], j] += Wx[i,j]*const[i] over i ascending, for `use` entries.

    `np.bincount` accumulates in input order, so each bin receives rows in
    ascending i, the reference's per-column order (algos.py:879-895)."""
    na, N = Wx.shape
    const = np.broadcast_to(np.asarray(const, np.float64).ravel(), (na,))
    V = Wx * const[:, None]
    out = np.empty((na, N), dtype=np.complex128)

    def block(j0, j1):
        kk = k[:, j0:j1]
        uu = use[:, j0:j1]
        cols = np.broadcast_to(np.arange(j1 - j0), kk.shape)
        lin = (kk * (j1 - j0) + cols)[uu]
        vv = V[:, j0:j1][uu]
        re = np.bincount(lin, weights=vv.real, minlength=na * (j1 - j0))
        im = np.bincount(lin, weights=vv.imag, minlength=na * (j1 - j0))
        out[:, j0:j1] = (re + 1j * im).reshape(na, j1 - j0)

    step = max(256, -(-N // (4 * _WORKERS)))
    spans = [(j, min(N, j + step)) for j in range(0, N, step)]
    if len(spans) == 1:
        block(*spans[0])
    else:
        with ThreadPoolExecutor(_WORKERS) as ex:
            list(ex.map(lambda s: block(*s), spans))
    return out


def ssq_cwt(x, kind, params, scales, ssq_freqs, const, dt=1.,
            padtype='reflect', logscale=True, flipud=True, gamma=None):
    """(Tx, Wx, w) of `ssq_cwt` for 1D or 2D `x`; `ssq_freqs` ascending, as
    passed to the squeeze (ssqueezing.py:122-146, 204-214)."""
    Wx, dWx = cwt(x, kind, params, scales, dt=dt, padtype=padtype)
    gamma = 10 * EPS64 if gamma is None else gamma
    if Wx.ndim == 2:
        w = phase_cwt(Wx, dWx, gamma)
        use = np.abs(Wx) > gamma
        k = bin_index(np.where(use, w, 1.), ssq_freqs, logscale, flipud)
        return squeeze(Wx, k, use, const), Wx, w
    outs = [ssq_cwt(xi_, kind, params, scales, ssq_freqs, const, dt, padtype,
                    logscale, flipud, gamma) for xi_ in x]
    return tuple(np.stack(o) for o in zip(*outs))


#### STFT (_stft.py:127-181, utils/stft_utils.py:20-98) #######################
def frames(xp, n_fft, hop, modulated=True):
    """(n_fft, n_frames) frame matrix; modulated frames are rotated by
    ceil(n_fft/2) (stft_utils.py:69-82)."""
    n_segs = (xp.shape[-1] - n_fft) // hop + 1
    s20 = int(np.ceil(n_fft / 2))
    s21 = s20 - 1 if n_fft % 2 == 1 else s20
    starts = hop * np.arange(n_segs)
    m = np.arange(n_fft)
    if modulated:
        src = np.where(m < s20, m + s21, m - s20)
    else:
        src = m
    return xp[..., starts[None, :] + src[:, None]]


def stft(x, window, diff_window, n_fft, hop=1, fs=1., padtype='reflect',
         modulated=True):
    """(Sx, dSx), each (n_fft//2+1, n_frames) (or batched)."""
    x = np.asarray(x, np.float64)
    N = x.shape[-1]
    padlength = N + n_fft - 1
    if abs(padlength - N) % 2 == 0:
        n1 = n2 = (padlength - N) // 2
    else:
        n2 = (padlength - N) // 2
        n1 = n2 + 1
    xp = pad(x, padtype, n1, n2)
    F = frames(xp, n_fft, hop, modulated)
    win = np.asarray(window, np.float64)
    dwin = np.asarray(diff_window, np.float64) * fs
    if modulated:
        win, dwin = np.fft.ifftshift(win), np.fft.ifftshift(dwin)
    ax = -2
    shp = (-1, 1)
    Sx = sfft.rfft(F * win.reshape(shp), axis=ax, workers=_WORKERS)
    dSx = sfft.rfft(F * dwin.reshape(shp), axis=ax, workers=_WORKERS)
    return Sx, dSx


def ssq_stft(x, window, diff_window, n_fft, hop=1, fs=1., padtype='reflect',
             modulated=True, flipud=False, gamma=None):
    """(Tx, Sx, w, Sfs) of `ssq_stft` (_ssq_stft.py:88-136)."""
    Sx, dSx = stft(x, window, diff_window, n_fft, hop, fs, padtype, modulated)
    gamma = 10 * EPS64 if gamma is None else gamma
    nrow = Sx.shape[-2]
    Sfs = np.linspace(0, .5 * fs, nrow)
    const = Sfs[1] - Sfs[0]
    if Sx.ndim == 2:
        w = phase_stft(Sx, dSx, Sfs, gamma)
        use = np.abs(Sx) > gamma
        k = bin_index(np.where(use, w, 0.), Sfs, False, flipud)
        return squeeze(Sx, k, use, const), Sx, w, Sfs
    outs = [ssq_stft(xi_, window, diff_window, n_fft, hop, fs, padtype,
                     modulated, flipud, gamma) for xi_ in x]
    Tx, S, w, _ = zip(*outs)
    return np.stack(Tx), np.stack(S), np.stack(w), Sfs


#### inverse CWT, one integral (_cwt.py:406-453, 479-494) #####################
def icwt(Wx, scales, scaletype, nv, Cpsi, x_mean=0., l1_norm=True):
    """x = (2/Cpsi) * sum over log pieces of (ln2/nv_p) sum_i Re Wx_i
    [/scale_i for linear] + x_mean; `nv` per row (log-piecewise) or scalar.

    For log-piecewise scales the reference recurses once per piece and each
    piece adds `x_mean` (_cwt.py:422-429, 452), so the mean enters twice."""
    scales = np.asarray(scales, np.float64).ravel()
    if scaletype == 'log-piecewise':
        idx = transition_idx(scales)
        nvs = np.asarray(nv, np.float64).ravel()
        return (icwt(Wx[..., :idx, :], scales[:idx], 'log', nvs[0], Cpsi,
                     x_mean, l1_norm) +
                icwt(Wx[..., idx:, :], scales[idx:], 'log', nvs[idx], Cpsi,
                     x_mean, l1_norm))
    if scaletype == 'log':
        norm = np.ones_like(scales) if l1_norm else scales**.5
    else:
        norm = scales if l1_norm else scales**1.5
    x = (Wx.real / norm.reshape(-1, 1)).sum(axis=-2)
    if scaletype == 'log':
        x = x * ((2 / Cpsi) * np.log(2 ** (1 / float(np.round(nv)))))
    else:
        x = x * ((2 / Cpsi) * PI / 4)
    return x + x_mean


#### adjoints (transposes of cwt, the squeeze and icwt) #######################
# ssqueezepy has no backward pass; these are the transposes of the forward
# routines above (cwt: _cwt.py:246-311; squeeze: algos.py:859-895 with bins
# held fixed; icwt: _cwt.py:479-482), used to check the adjoint kernels.
# Gradients follow torch's complex convention g = dL/dRe + i dL/dIm, so for
# a real x, Re <g, cwt(x)> = <x, cwt_adjoint(g)>.
def pad_sources(N, padtype, n1, n2):
    """Source sample of each padded position; -1 where the padding is zero."""
    src = pad(np.arange(1, N + 1, dtype=np.float64), padtype, n1, n2)
    return np.rint(src).astype(np.int64) - 1


def cwt_adjoint(g, kind, params, scales, padtype='reflect'):
    """Gradient of x (..., N) for a gradient g (..., na, N) of Wx."""
    g = np.asarray(g, np.complex128)
    N = g.shape[-1]
    Npad, n1, n2 = p2up(N)
    gp = np.zeros(g.shape[:-1] + (Npad,), np.complex128)
    gp[..., n1:n1 + N] = g
    H = sfft.fft(gp, axis=-1, workers=_WORKERS)
    P, _ = psih_bank(kind, params, scales, Npad)
    yp = sfft.ifft((P * H).sum(axis=-2), axis=-1, workers=_WORKERS).real
    src = pad_sources(N, padtype, n1, n2)
    keep = src >= 0
    yp2 = yp.reshape(-1, Npad)
    out = np.zeros((yp2.shape[0], N))
    for b in range(yp2.shape[0]):
        np.add.at(out[b], src[keep], yp2[b, keep])
    return out.reshape(g.shape[:-2] + (N,))


def squeeze_adjoint(gT, k, use, const):
    """Gradient of Wx (na, N) for a gradient gT (na, N) of Tx: the gather
    const[i] * gT[k[i, j], j] where `use`, else 0."""
    na, N = k.shape
    const = np.broadcast_to(np.asarray(const, np.float64).ravel(), (na,))
    cols = np.broadcast_to(np.arange(N), k.shape)
    return np.where(use, gT[k, cols] * const[:, None], 0)


def icwt_adjoint(gx, weights):
    """Gradient of Wx (..., na, N) for a gradient gx (..., N) of
    x = sum_i weights[i] Re Wx[i] (+ mean): weights[i] * gx (real)."""
    w = np.asarray(weights, np.float64).reshape(-1, 1)
    return (w * np.asarray(gx, np.float64)[..., None, :]).astype(np.complex128)


def stft_adjoint(gS, window, n_fft, N, hop=1, padtype='reflect', modulated=True):
    """Gradient of x (..., N) for a gradient gS (..., n_fft//2+1, n_frames)
    of Sx = stft(x)[0] (the transpose of `frames`, the window and `rfft`)."""
    gS = np.asarray(gS, np.complex128)
    L = n_fft
    nfr = gS.shape[-1]
    G = np.zeros(gS.shape[:-2] + (L, nfr), np.complex128)
    G[..., :L // 2 + 1, :] = gS
    gu = (sfft.ifft(G, axis=-2, workers=_WORKERS) * L).real   # (..., L, n_frames)
    win = np.asarray(window, np.float64)
    if modulated:
        win = np.fft.ifftshift(win)
    gF = gu * win.reshape(-1, 1)
    padlength = N + n_fft - 1
    if abs(padlength - N) % 2 == 0:
        n1 = n2 = (padlength - N) // 2
    else:
        n2 = (padlength - N) // 2
        n1 = n2 + 1
    s20 = int(np.ceil(n_fft / 2))
    s21 = s20 - 1 if n_fft % 2 == 1 else s20
    m = np.arange(n_fft)
    srcm = np.where(m < s20, m + s21, m - s20) if modulated else m
    pos = hop * np.arange(nfr)[None, :] + srcm[:, None]            # padded position
    src = pad_sources(N, padtype, n1, n2)
    gF2 = gF.reshape(-1, L, nfr)
    out = np.zeros((gF2.shape[0], N))
    for b in range(gF2.shape[0]):
        gxp = np.zeros(padlength)
        np.add.at(gxp, pos.ravel(), gF2[b].ravel())
        keep = src >= 0
        np.add.at(out[b], src[keep], gxp[keep])
    return out.reshape(gS.shape[:-2] + (N,))


#### inverse synchrosqueezing (_ssq_cwt.py:313-400, _ssq_stft.py:139-198) ####
def istft(Sx, window, n_fft, hop=1, N=None, modulated=True, win_exp=1):
    """Inverse STFT of one-sided `Sx` (n_fft//2+1, n_frames) with the
    n_fft-long `window` (_stft.py:184-256): irfft per frame, fftshift when
    modulated, overlap-add with window^win_exp (utils/stft_utils.py:141-182),
    divide by the window norm of window^(win_exp+1) over (N-1)//hop + 1 hops
    (:169-191) where it exceeds the data type's tiny, unpad n_fft//2 on the
    left. Arithmetic in the window's dtype, as the reference."""
    nframes = Sx.shape[1]
    N = N or hop * nframes
    dtype = np.float32 if Sx.dtype == np.complex64 else np.float64
    window = np.asarray(window).astype(dtype)
    xbuf = np.fft.irfft(Sx, n=n_fft, axis=0).astype(dtype)
    if modulated:
        xbuf = np.fft.fftshift(xbuf, axes=0)
    wa = np.ones_like(window) if win_exp == 0 else window ** win_exp
    Lx = N + n_fft - 1
    x = np.zeros(Lx, dtype=dtype)
    for i in range(nframes):
        x[i * hop:i * hop + n_fft] += xbuf[:, i] * wa
    wn = np.zeros(Lx)
    w1 = window ** (win_exp + 1)
    for i in range((Lx - n_fft) // hop + 1):
        wn[i * hop:i * hop + n_fft] += w1
    th = np.finfo(dtype).tiny
    keep = wn > th
    x[keep] = x[keep] / wn[keep]
    return x[n_fft // 2:Lx - (n_fft - 1) // 2]


def issq(Tx, scale, cc=None, cw=None):
    """scale * sum_k Re Tx[k] (full inversion) or, with curve centres `cc` and
    widths `cw` (N, K), the K components summed over their row bands
    [clip(cc - cw), clip(cc + cw)] (empty where cc = -1) and, last, the rows
    outside every band: (K + 1, N) float64."""
    Tx = np.asarray(Tx)
    if cc is None and cw is None:
        return Tx.real.sum(axis=0) * scale
    cc = np.asarray(cc).reshape(len(cc), -1).astype(np.int32)
    cw = np.asarray(cw).reshape(len(cw), -1).astype(np.int32)
    nr, N = Tx.shape
    K = cc.shape[1]
    x = np.zeros((K + 1, N))
    keep = np.ones(Tx.shape, bool)
    for n in range(K):
        up = np.clip(cc[:, n] + cw[:, n], 0, nr)
        lo = np.clip(cc[:, n] - cw[:, n], 0, nr)
        up[cc[:, n] == -1] = 0
        lo[cc[:, n] == -1] = 1
        rows = np.arange(nr)[:, None]
        band = (rows >= lo[None, :]) & (rows <= up[None, :])
        x[n] = np.where(band, Tx.real, 0).sum(axis=0)
        keep &= ~band
    x[K] = np.where(keep, Tx.real, 0).sum(axis=0)
    return x * scale


#### ridge extraction (ridge_extraction.py:11-232, serial code path) ##########
def ridge_track(E, P, eps):
    """Forward min-plus sweep of E (nf, N) with jump penalties P (nf, nf),
    then the backward re-tracking: the last row whose accumulated value
    reproduces within eps, else the column's argmin (ridge_extraction.py:
    147-162, 187-232), in E's arithmetic type."""
    N = E.shape[1]
    pen = E.copy()
    for t in range(1, N):
        pen[:, t] += np.amin(pen[:, t - 1][None, :] + P, axis=1)
    r = np.argmin(pen, axis=0)
    for t in range(N - 2, -1, -1):
        val = pen[r[t + 1], t + 1] - E[r[t + 1], t + 1]
        hit = np.nonzero(np.abs(val - (pen[:, t] + P[r[t + 1], :])) < eps)[0]
        if len(hit):
            r[t] = hit[-1]
    return r


def extract_ridges(Tf, scales, penalty=2., n_ridges=1, bw=15, transform='cwt'):
    """(ridge_idxs, ridge_f, ridge_e), each (N, n_ridges): forward-backward
    tracking of min accumulated -log normalised energy plus
    penalty * (s_f - s_f')^2 jumps (s = log scales for 'cwt'), in the
    arithmetic type of Tf (float32 for complex64)."""
    Tf = np.asarray(Tf)
    dt = np.float64 if Tf.dtype == np.complex128 else np.float32
    eps = dt(EPS64 if dt == np.float64 else EPS32)
    scales = np.asarray(scales, dt)
    penalty = dt(penalty)
    s = (np.log(scales) if transform == 'cwt' else scales).squeeze()
    P = penalty * np.subtract.outer(s, s) ** 2
    energy = np.abs(Tf) ** 2
    nf, N = energy.shape
    idxs = np.zeros((N, n_ridges), int)
    rf = np.zeros((N, n_ridges), dt)
    re = np.zeros((N, n_ridges), dt)
    for i in range(n_ridges):
        E = -np.log(energy / energy.max(axis=0) + eps)
        r = ridge_track(E, P, eps)
        idxs[:, i] = r
        rf[:, i] = scales[r]
        re[:, i] = energy[r, np.arange(N)]
        for t in range(N):
            energy[int(r[t] - bw):int(r[t] + bw), t] = 0
    return idxs, rf, re
