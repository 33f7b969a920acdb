# -*- coding: utf-8 -*-
"""Drop-in `cwt`, `ssq_cwt`, `icwt`, `stft`, `ssq_stft`, `ssqueeze` on the
GPU. Signatures and return tuples follow ssqueezepy (paths relative to its
source tree): `ssq_cwt` _ssq_cwt.py:12-310, `cwt` _cwt.py:12-320, `icwt`
_cwt.py:323-453, `stft` _stft.py:13-181, `ssq_stft` _ssq_stft.py:13-136,
`ssqueeze` ssqueezing.py:13-224.

Host work is the float64 parameter math of `_params`; every array operation
runs in the CUDA kernels of libssqb.so (through `_lib`). Inputs may be numpy
arrays or torch tensors (CPU or CUDA); outputs are CUDA tensors
(`astensor=True`, the default) or numpy arrays.
"""
import os
import warnings

import numpy as np
import torch

from . import _autograd as A
from . import _lib as L
from . import _params as P

__all__ = ['cwt', 'ssq_cwt', 'icwt', 'stft', 'ssq_stft', 'ssqueeze',
           'phase_cwt', 'phase_stft', 'issq_cwt', 'issq_stft', 'Wavelet', 'configure']

Wavelet = P.Wavelet

_CDT = {'float32': torch.complex64, 'float64': torch.complex128}
_RDT = {'float32': torch.float32, 'float64': torch.float64}


#### helpers #################################################################
def _device_of(x):
    if isinstance(x, torch.Tensor) and x.is_cuda:
        return x.device
    return torch.device('cuda', torch.cuda.current_device())


def _to_device(x, dtype, nan_checks):
    """(B, N) contiguous CUDA tensor of `dtype` and whether x was 2D."""
    if not hasattr(x, 'ndim'):
        raise TypeError("`x` must be a numpy array or torch Tensor "
                        "(got %s)" % type(x))
    if x.ndim not in (1, 2):
        raise ValueError("`x` must be 1D or 2D (got x.ndim == %s)" % x.ndim)
    L.require_cuda()
    is_np = isinstance(x, np.ndarray)
    if nan_checks is None:
        nan_checks = is_np
    if nan_checks:
        if not is_np:
            raise ValueError("`nan_checks=True` requires NumPy input.")
        if not np.isfinite(x).all():  # _cwt.py:208-215 zeroes NaN / inf
            x = np.where(np.isfinite(x), x, 0)
    dev = _device_of(x)
    t = torch.as_tensor(x)
    t = t.to(device=dev, dtype=_RDT[dtype], non_blocking=True)
    is_2d = t.ndim == 2
    return t.reshape(-1, t.shape[-1]).contiguous(), is_2d


def _out(t, astensor, is_2d=True):
    if t is None:
        return None
    if not is_2d and t.ndim >= 1 and t.shape[0] == 1:
        t = t[0]
    if astensor:
        return t
    return t.cpu().numpy()


# Arithmetic of float32 transforms: 'float64' (default) computes the FFTs,
# phase transform and bins in float64 and stores float32, so bins match the
# float64 path; 'float32' is faster and matches the reference's own float32
# path in accuracy (Tx differs from float64 at ~1e-3 relative L2 through bin
# flips).
_CONFIG = {'float32_arithmetic': os.environ.get('SSQB_FLOAT32_ARITHMETIC',
                                                'float64')}


def configure(float32_arithmetic=None):
    """Set the arithmetic of float32 transforms ('float64' or 'float32');
    returns the current settings."""
    if float32_arithmetic is not None:
        if float32_arithmetic not in ('float64', 'float32'):
            raise ValueError("`float32_arithmetic` must be 'float64' or 'float32'")
        _CONFIG['float32_arithmetic'] = float32_arithmetic
    return dict(_CONFIG)


def _prec(dtype):
    if dtype == 'float64':
        return L.F64
    return L.F32 if _CONFIG['float32_arithmetic'] == 'float32' else L.F32X


def _default_gamma(dtype):
    return 10 * (P.EPS64 if dtype == 'float64' else P.EPS32)


def _dev_f64(a, dev):
    # a copy: read-only inputs (np.load, broadcast views) give writable memory
    return torch.as_tensor(np.array(a, dtype=np.float64).ravel(), device=dev)


#### host parameter cache ###################################################
# The scale and frequency searches cost milliseconds of host time; a given
# (wavelet, N, scheme) always yields the same float64 parameters, so they are
# computed once. Device copies are kept per device.
_PLANS = {}
_PLAN_MAX = 1024


def _wkey(wavelet):
    return (wavelet.name_, tuple(sorted(wavelet.config.items())), wavelet.dtype)


def _akey(a):
    if a is None or isinstance(a, (str, int, float, tuple)):
        return a
    a = np.ascontiguousarray(P._to_numpy(a))
    return (a.dtype.str, a.shape, a.tobytes())


def _plan(key, make):
    p = _PLANS.get(key)
    if p is None:
        if len(_PLANS) >= _PLAN_MAX:
            _PLANS.pop(next(iter(_PLANS)))
        p = _PLANS[key] = make()
        p['dev'] = {}
    return p


def _on_device(plan, name, dev):
    k = (name, str(dev))
    t = plan['dev'].get(k)
    if t is None:
        t = plan['dev'][k] = _dev_f64(plan[name], dev)
    return t


def _scales_plan(scales, N, wavelet, nv):
    def make():
        if isinstance(scales, str):
            sc, st, na, nv_ = P.process_scales(scales, N, wavelet, nv=nv,
                                               get_params=True)
        else:
            sc, st, na, nv_ = P.process_scales(P._to_numpy(scales), N,
                                               get_params=True)
        # `scales_in` keeps the caller's dtype: inferring the scale type of
        # float32 scales takes float32 tolerances (cwt_utils.py:375-394)
        return dict(scales=np.asarray(sc, np.float64).ravel(), scaletype=st,
                    na=na, nv=nv_, scales_in=np.asarray(sc).reshape(-1, 1))
    return _plan(('scales', _wkey(wavelet), N, _akey(scales), nv), make)


#### CWT #####################################################################
def _cwt_core(x, wavelet, scales, nv, fs, t, padtype, rpadded, nan_checks,
              derivative, want_idx=False, want_w=False, ssq=None, gamma=None,
              kernel=None):
    """Run the fused CWT kernel. Returns dict of device tensors + params.
    `kernel` (default `wavelet`) is the wavelet the transform evaluates; a
    higher-order GMW transform takes its scales from the order-0 wavelet."""
    N = x.shape[-1]
    dt, fs, _ = P.process_fs_and_t(fs, t, N)
    wavelet = P.Wavelet._init_if_not_isinstance(wavelet)
    dtype = wavelet.dtype
    xd, is_2d = _to_device(x, dtype, nan_checks)
    dev = xd.device
    sp = _scales_plan(scales, N, wavelet, nv)
    scales_np, scaletype, na, nv = sp['scales'], sp['scaletype'], sp['na'], sp['nv']
    if padtype is None:
        Npad, n1 = N, 0
        if Npad & (Npad - 1):
            raise NotImplementedError("`padtype=None` needs a power-of-2 length "
                                      "on the accelerated path")
        ptype = 5
    else:
        if padtype not in L.PADTYPES:
            raise ValueError("`padtype` must be one of %s (got %s)"
                             % (list(L.PADTYPES), padtype))
        Npad, n1, _ = P.p2up(N)
        ptype = L.PADTYPES[padtype]
    B = xd.shape[0]
    ncol = Npad if (rpadded and padtype is not None) else N
    prec = _prec(dtype)
    cdt, rdt = _CDT[dtype], _RDT[dtype]
    Wx = torch.empty((B, na, ncol), dtype=cdt, device=dev)
    dWx = torch.empty_like(Wx) if derivative else None
    w = torch.empty((B, na, ncol), dtype=rdt, device=dev) if want_w else None
    ipitch = L.idx_pitch(ncol)
    idx = (torch.empty((B, na, ipitch), dtype=torch.uint16, device=dev)
           if want_idx else None)
    wsb = L.load().ssqb_cwt_workspace_bytes(B, N, Npad, na, prec)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    sc_d = _on_device(sp, 'scales', dev)
    cw = L.wavelet_struct(kernel or wavelet)
    cb = L.make_bins(*ssq) if ssq is not None else None
    gamma = _default_gamma(dtype) if gamma is None else gamma
    sc_h = np.ascontiguousarray(scales_np, np.float64)  # lets the call plan per row
    with torch.cuda.device(dev):
        rc = L.load().ssqb_cwt_ex(
            L.ptr(xd), B, N, Npad, n1, ptype, 1 if (rpadded and padtype) else 0,
            L.ptr(sc_d), sc_h.ctypes.data, na, cw, float(dt), cb, float(gamma), prec,
            L.ptr(Wx), L.ptr(dWx), L.ptr(w), L.ptr(idx), ipitch, L.ptr(ws), wsb,
            L.stream_ptr())
    L.check(rc, 'cwt')
    return dict(Wx=Wx, dWx=dWx, w=w, idx=idx, ipitch=ipitch, scales=scales_np,
                scaletype=scaletype, nv=nv, na=na, N=N, dt=dt, fs=fs,
                wavelet=wavelet, dtype=dtype, is_2d=is_2d, dev=dev, B=B,
                gamma=gamma, sc_d=sc_d, Npad=Npad, n1=n1, ptype=ptype, cw=cw,
                prec=prec)


def cwt(x, wavelet='gmw', scales='log-piecewise', fs=None, t=None, nv=32,
        l1_norm=True, derivative=False, padtype='reflect', rpadded=False,
        vectorized=True, astensor=True, cache_wavelet=None, order=0, average=None,
        nan_checks=None, patience=0):
    """Continuous Wavelet Transform; returns `(Wx, scales[, dWx])`
    (_cwt.py:12-320). `vectorized`, `cache_wavelet` and `patience` only
    select CPU strategies in the reference and have no effect here."""
    if isinstance(order, (tuple, list, range)) or order > 0:
        return _cwt_higher_order(x, wavelet, order, average, astensor, dict(
            scales=scales, fs=fs, t=t, nv=nv, l1_norm=l1_norm,
            derivative=derivative, padtype=padtype, rpadded=rpadded,
            nan_checks=nan_checks))
    if not isinstance(scales, str):
        nv = None
    wavelet = P.process_gmw_wavelet(wavelet, l1_norm)

    def run(xin):
        return _cwt_core(xin, wavelet, scales, nv, fs, t, padtype, rpadded, nan_checks,
                         derivative)
    if A.needs_grad(x):
        _grad_checks(astensor, rpadded and padtype is not None, padtype)
        holder = {}

        def run_keep(xin):
            holder['r'] = run(xin)
            return holder['r']
        outs = A.CwtFn.apply(x, run_keep)
        r = holder['r']
        Wx, dWx = (outs if derivative else (outs, None))
    else:
        r = run(x)
        Wx, dWx = r['Wx'], r['dWx']
    if not l1_norm:
        s = torch.as_tensor(np.sqrt(r['scales'].ravel()), device=r['dev'],
                            dtype=_RDT[r['dtype']]).reshape(1, -1, 1)
        Wx = Wx * s
        dWx = dWx * s if dWx is not None else None
    scales_out = _scales_out(r, astensor)
    Wx, dWx = _out(Wx, astensor, r['is_2d']), _out(dWx, astensor, r['is_2d'])
    return (Wx, scales_out, dWx) if derivative else (Wx, scales_out)


def _gmw_options(wavelet, N):
    """The options of a GMW `wavelet` without its order, for building its
    other orders (cwt_higher_order, _cwt.py:551-560)."""
    base = P.Wavelet._init_if_not_isinstance(wavelet, N=N)
    if not base.name.lower().startswith('gmw'):
        raise ValueError("`wavelet` must be GMW for higher-order transforms "
                         "(got %s)" % base.name)
    opts = dict(base.config, dtype=base.dtype)
    opts.pop('order', None)
    return opts


def _order0_scales(scales, N, opts, nv):
    """String scales of a higher-order transform come from the order-0
    wavelet (_cwt.py:573-578); an array passes through."""
    if not isinstance(scales, str):
        return scales
    wav0 = P.Wavelet(('gmw', dict(opts, order=0)))
    return _scales_plan(scales, N, wav0, nv)['scales'].reshape(-1, 1)


def _cwt_higher_order(x, wavelet, order, average, astensor, kw):
    """`cwt` with higher-order GMWs (cwt_higher_order, _cwt.py:517-610).
    The transform is linear in the wavelet, so the mean over orders is one
    transform with the mean wavelet, whose Laguerre coefficients are the
    mean of the orders' (`Wavelet.poly`); `average=False` runs one transform
    per order and returns lists. Scales come back as a column (na, 1), as
    the reference returns them on this path."""
    if isinstance(order, (list, range)):
        order = tuple(order)
    orders = order if isinstance(order, tuple) else (order,)
    P._check_order(orders)
    if len(orders) == 1 and average:
        warnings.warn("`average` ignored with single `order`")
        average = False
    N = x.shape[-1]
    opts = _gmw_options(wavelet, N)
    scales = _order0_scales(kw.pop('scales'), N, opts, kw['nv'])
    avg = average or (average is None and isinstance(order, tuple))
    groups = [orders] if avg else [(k,) for k in orders]
    outs = [cwt(x, P.Wavelet(('gmw', dict(opts, order=g))), scales=scales, order=0,
                astensor=astensor, **kw) for g in groups]
    derivative = kw['derivative']
    Wx = [o[0] for o in outs]
    dWx = [o[-1] for o in outs] if derivative else None
    if len(outs) == 1:
        Wx = Wx[0]
        dWx = dWx[0] if derivative else None
    sc = outs[0][1].reshape(-1, 1)
    return (Wx, sc, dWx) if derivative else (Wx, sc)


def _grad_checks(astensor, rpadded, padtype):
    if not astensor:
        raise ValueError("differentiable transforms return tensors: use astensor=True")
    if rpadded:
        raise NotImplementedError("gradients of `rpadded=True` outputs are not "
                                  "implemented")
    if padtype == 'replicate':
        raise NotImplementedError("gradients through padtype='replicate' are not "
                                  "implemented")


def _scales_out(r, astensor):
    if astensor:
        # a device-side cast of the cached float64 scales: no host copy, so
        # the call stays asynchronous
        return r['sc_d'].to(_RDT[r['dtype']], copy=True)
    return r['scales'].ravel().astype(r['dtype'])


def _check_ssq_args(squeezing, maprange, difftype, get_w=True, difforder=None):
    """The argument checks of ssqueezing.py:314-368; returns `difforder`
    (4 by default for difftype='numeric')."""
    if not (isinstance(squeezing, str) or callable(squeezing)):
        raise TypeError("`squeezing` must be string or function "
                        "(got %s)" % type(squeezing))
    if isinstance(squeezing, str) and squeezing not in ('sum', 'lebesgue', 'abs'):
        raise ValueError("`squeezing` must be one of: sum, lebesgue, abs "
                         "(got %s)" % squeezing)
    if isinstance(maprange, (tuple, list)):
        if not all(isinstance(m, (float, int)) for m in maprange):
            raise ValueError("all elements of `maprange` must be float or int")
    elif isinstance(maprange, str):
        if maprange not in ('maximal', 'peak', 'energy'):
            raise ValueError("`maprange` must be one of: maximal, peak, energy "
                             "(got %s)" % maprange)
    else:
        raise TypeError("`maprange` must be str, tuple, or list "
                        "(got %s)" % type(maprange))
    if difftype not in ('trig', 'phase', 'numeric'):
        raise ValueError("`difftype` must be one of: direct, phase, numeric"
                         " (got %s)" % difftype)
    if difftype != 'trig' and not get_w:
        raise ValueError("`difftype != 'trig'` requires `get_w = True`")
    if difforder is not None:
        if difftype != 'numeric':
            warnings.warn("`difforder` is ignored if `difftype != 'numeric'")
        elif difforder not in (1, 2, 4):
            raise ValueError("`difforder` must be one of: 1, 2, 4 "
                             "(got %s)" % difforder)
    elif difftype == 'numeric':
        difforder = 4
    return difforder


def _squeeze_values(W, squeezing):
    """The values the squeeze sums (ssqueezing.py:196-201): Wx itself for
    'sum', `ones / len(Wx)` for 'lebesgue' (len: the first axis of Wx as the
    caller shaped it), |Wx| for 'abs', or `squeezing(Wx)` for a function (on
    the device tensor). With no `w` given, the reference also takes the phase
    transform from these values and dWx, and so does the squeeze here."""
    if callable(squeezing):
        out = torch.as_tensor(squeezing(W)).to(device=W.device, dtype=W.dtype)
        if out.shape != W.shape:
            raise ValueError("`squeezing` function must keep the shape of Wx")
        return out.contiguous()
    if squeezing == 'lebesgue':
        return torch.full_like(W, 1. / W.shape[0])
    if squeezing == 'abs':
        return W.abs().to(W.dtype)
    return W


def _squeeze_from(Wv, w, dW, sfs_d, cst, mode, bp, nbins, flipud, gamma):
    """Tx from squeeze values Wv (B, na, N) and either a phase transform w
    (`ssqb_indexed_sum`) or dWx for the phase on the fly
    (`ssqb_ssqueeze_fast`)."""
    B, na, N = Wv.shape
    prec = L.F64 if Wv.dtype == torch.complex128 else L.F32
    Tx = torch.empty_like(Wv)
    cb = L.make_bins(mode, bp, nbins, flipud)
    with torch.cuda.device(Wv.device):
        if w is not None:
            rc = L.load().ssqb_indexed_sum(L.ptr(Wv), L.ptr(w.contiguous()), L.ptr(cst), cb,
                                           B, na, N, prec, L.ptr(Tx), L.stream_ptr())
        else:
            rc = L.load().ssqb_ssqueeze_fast(L.ptr(Wv), L.ptr(dW.contiguous()), L.ptr(sfs_d),
                                             L.ptr(cst), cb, float(gamma), B, na, N, prec,
                                             L.ptr(Tx), L.stream_ptr())
    L.check(rc, 'ssqueeze')
    return Tx


def _ssq_freqs_for_cwt(ssq_freqs, scales, N, wavelet, cwt_scaletype, maprange,
                       was_padded, dt):
    """Ascending ssq_freqs (float64) and whether bins are log-spaced
    (ssqueezing.py:168-194)."""
    if isinstance(ssq_freqs, (np.ndarray, torch.Tensor)):
        f = P._to_numpy(ssq_freqs).astype(np.float64).ravel()
        st, _ = P.infer_scaletype(f)
        return f, st.startswith('log')
    st = ssq_freqs if isinstance(ssq_freqs, str) else cwt_scaletype
    if ((maprange == 'maximal' or isinstance(maprange, tuple)) and
            st == 'log-piecewise'):
        raise ValueError("can't have `ssq_scaletype = log-piecewise` or "
                         "tuple with `maprange = 'maximal'` "
                         "(got %s)" % str(maprange))
    f = P.compute_associated_frequencies(scales, N, wavelet, st, maprange,
                                         was_padded, dt, 'cwt')
    return np.asarray(f, np.float64), st.startswith('log')


def _ssq_plan(wavelet, scales, N, nv, ssq_freqs, maprange, padtype, dt, sp=None):
    """Host parameters of the squeeze of `ssq_cwt`: ascending ssq_freqs, bin
    mapping and per-row weights (float64, cached)."""
    sp = sp or _scales_plan(scales, N, wavelet, nv)
    sc, cwt_st = sp['scales'], sp['scaletype']

    def make():
        f_asc, logscale = _ssq_freqs_for_cwt(
            ssq_freqs, sp['scales_in'], N, wavelet, cwt_st, maprange,
            padtype is not None, dt)
        mode, bp = P.bin_params(f_asc, logscale)
        # ssqueeze re-derives (scaletype, nv) from the scale array, so a
        # log-piecewise grid gets ln2/nv per row (ssqueezing.py:168-169, 124-128)
        _, st_a, _, nv_a = P.process_scales(sp['scales_in'], N, get_params=True)
        const = P.squeeze_weights(sc, st_a, nv_a, 'cwt')
        return dict(f_asc=f_asc, mode=mode, bp=bp, const=const)
    return _plan(('ssq', _wkey(wavelet), N, _akey(scales), nv, _akey(ssq_freqs),
                  _akey(maprange), padtype is not None, dt), make)


def ssq_cwt(x, wavelet='gmw', scales='log-piecewise', nv=None, fs=None, t=None,
            ssq_freqs=None, padtype='reflect', squeezing='sum', maprange='peak',
            difftype='trig', difforder=None, gamma=None, vectorized=True,
            preserve_transform=None, astensor=True, order=0, nan_checks=None,
            patience=0, flipud=True, cache_wavelet=None, get_w=False,
            get_dWx=False):
    """Synchrosqueezed CWT; returns `(Tx, Wx, ssq_freqs, scales[, w][, dWx])`
    (_ssq_cwt.py:12-310). `ssq_freqs` comes back as a float64 numpy array,
    high to low (ssqueezing.py:216-224)."""
    if x.ndim == 2 and get_w:
        raise NotImplementedError("`get_w=True` unsupported with batched input.")
    difforder = _check_ssq_args(squeezing, maprange, difftype, get_w, difforder)
    if nv is None and not isinstance(scales, np.ndarray):
        nv = 32
    N = x.shape[-1]
    dt, fs, _ = P.process_fs_and_t(fs, t, N)
    wavelet = P.Wavelet._init_if_not_isinstance(wavelet, N=N)
    kernel = None
    if isinstance(order, (tuple, list, range)) or order > 0:
        # higher-order GMW (_ssq_cwt.py:227-243): the transform with the mean
        # wavelet of a tuple of orders, or with order k alone; its derivative
        # (the reference's trigdiff of the padded transform) is the same
        # frequency-domain derivative the fused kernel takes. The squeeze keeps
        # the user's wavelet for `maprange`.
        if isinstance(order, (list, range)):
            order = tuple(order)
        P._check_order(order)
        opts = _gmw_options(wavelet, N)
        scales = _order0_scales(scales, N, opts, nv)
        kernel = P.Wavelet(('gmw', dict(opts, order=order)))
    sp = _scales_plan(scales, N, wavelet, nv)
    sc, cwt_st, na, nv_ = sp['scales'], sp['scaletype'], sp['na'], sp['nv']

    if difftype != 'trig':
        return _ssq_cwt_by_differences(
            x, wavelet, kernel, scales, nv, fs, t, dt, padtype, nan_checks, gamma, sp,
            ssq_freqs, maprange, flipud, difftype, difforder, astensor, get_dWx,
            squeezing)
    if not (isinstance(squeezing, str) and squeezing == 'sum'):
        # the squeeze sums other values than Wx (ssqueezing.py:196-201): Wx
        # and dWx (or w) first, then the squeeze from the replaced values
        if A.needs_grad(x):
            raise NotImplementedError("gradients need squeezing='sum'")
        fp = _ssq_plan(wavelet, scales, N, nv, ssq_freqs, maprange, padtype, dt, sp)
        r = _cwt_core(x, wavelet, scales, nv, fs, t, padtype, False, nan_checks, True,
                      want_w=get_w, gamma=gamma, kernel=kernel)
        is2 = r['is_2d']
        W3 = r['Wx']
        Wv = _squeeze_values(W3 if is2 else W3[0], squeezing)
        Wv = Wv if is2 else Wv[None]
        Tx = _squeeze_from(Wv, r['w'], r['dWx'], None, _on_device(fp, 'const', r['dev']),
                           fp['mode'], fp['bp'], na, flipud, r['gamma'])
        out = [_out(Tx, astensor, is2), _out(W3, astensor, is2), fp['f_asc'][::-1],
               _scales_out(r, astensor)]
        if get_w:
            out.append(_out(r['w'], astensor, is2))
        if get_dWx:
            out.append(_out(r['dWx'], astensor, is2))
        return tuple(out)
    fp = _ssq_plan(wavelet, scales, N, nv, ssq_freqs, maprange, padtype, dt, sp)
    f_asc = fp['f_asc']
    def run(xin):
        r = _cwt_core(xin, wavelet, scales, nv, fs, t, padtype, False, nan_checks,
                      get_dWx, want_idx=True, want_w=get_w,
                      ssq=(fp['mode'], fp['bp'], na, flipud), gamma=gamma,
                      kernel=kernel)
        Tx = torch.empty_like(r['Wx'])
        cst = _on_device(fp, 'const', r['dev'])
        with torch.cuda.device(r['dev']):
            rc = L.load().ssqb_squeeze(L.ptr(r['Wx']), L.ptr(r['idx']), r['ipitch'],
                                       L.ptr(cst), r['B'], na, N, na, _prec(r['dtype']),
                                       L.ptr(Tx), L.stream_ptr())
        L.check(rc, 'squeeze')
        return Tx, r, cst

    if A.needs_grad(x):
        _grad_checks(astensor, False, padtype)
        holder = {}

        def run_keep(xin):
            holder['out'] = run(xin)
            return holder['out']
        Tx, Wx = A.SsqCwtFn.apply(x, run_keep)
        r = holder['out'][1]
    else:
        Tx, r, _ = run(x)
        Wx = r['Wx']
    is2 = r['is_2d']
    out = [_out(Tx, astensor, is2), _out(Wx, astensor, is2), f_asc[::-1],
           _scales_out(r, astensor)]
    if get_w:
        out.append(_out(r['w'], astensor, is2))
    if get_dWx:
        out.append(_out(r['dWx'], astensor, is2))
    return tuple(out)


def _ssq_cwt_by_differences(x, wavelet, kernel, scales, nv, fs, t, dt, padtype,
                            nan_checks, gamma, sp, ssq_freqs, maprange, flipud,
                            difftype, difforder, astensor, get_dWx, squeezing='sum'):
    """`ssq_cwt` with difftype 'phase' or 'numeric' (get_w=True): the phase
    transform from differences of Wx along time (`ssqb_phase_diff`), then the
    squeeze from it (`ssqb_indexed_sum`). 'numeric' works on the padded
    transform's columns n1-4 .. n1+N+3, its squeeze sees those N+8 columns,
    and 4 columns are trimmed from each side of Tx, w and the padded Wx
    afterwards, as in _ssq_cwt.py:205-220, 246-300."""
    if A.needs_grad(x):
        raise NotImplementedError("gradients with difftype != 'trig' are not "
                                  "implemented")
    numeric = difftype == 'numeric'
    if numeric and padtype is None:
        raise NotImplementedError("difftype='numeric' needs a padded transform "
                                  "(`padtype` not None)")
    N = x.shape[-1]
    r = _cwt_core(x, wavelet, scales, nv, fs, t, padtype, numeric, nan_checks,
                  get_dWx, gamma=gamma, kernel=kernel)
    W, B, na, dev = r['Wx'], r['B'], r['na'], r['dev']
    col0, M = (r['n1'] - 4, N + 8) if numeric else (0, N)
    fp = _ssq_plan(wavelet, scales, M, nv, ssq_freqs, maprange, padtype, dt, sp)
    prec = L.F64 if r['dtype'] == 'float64' else L.F32
    w = torch.empty((B, na, M), dtype=_RDT[r['dtype']], device=dev)
    lib = L.load()
    with torch.cuda.device(dev):
        rc = lib.ssqb_phase_diff(L.ptr(W), B, na, W.shape[-1], col0, M,
                                 2 if numeric else 1, int(difforder or 4), float(dt),
                                 float(r['gamma']), prec, L.ptr(w), L.stream_ptr())
        L.check(rc, 'phase_diff')
        Ws = W[..., col0:col0 + M].contiguous() if numeric else W
    is2 = r['is_2d']
    Wv = _squeeze_values(Ws if is2 else Ws[0], squeezing)
    Tx = _squeeze_from(Wv if is2 else Wv[None], w, None, None,
                       _on_device(fp, 'const', dev), fp['mode'], fp['bp'], na, flipud, 0.)
    if numeric:
        # Tx and w lose the 4 extra columns each side; the returned Wx is the
        # padded transform less 4 columns each side (_ssq_cwt.py:294-296)
        Ws, Tx, w = (a[..., 4:-4].contiguous() for a in (W, Tx, w))
    out = [_out(Tx, astensor, is2), _out(Ws, astensor, is2), fp['f_asc'][::-1],
           _scales_out(r, astensor), _out(w, astensor, is2)]
    if get_dWx:
        out.append(_out(r['dWx'], astensor, is2))
    return tuple(out)


def icwt(Wx, wavelet='gmw', scales='log-piecewise', nv=None, one_int=True,
         x_len=None, x_mean=0, padtype='reflect', rpadded=False, l1_norm=True):
    """One-integral inverse CWT (_cwt.py:323-453) as one weighted row sum on
    the GPU. `Wx` (na, n) or (B, na, n); returns (n,) or (B, n), same
    container kind as `Wx`."""
    if not one_int:
        raise NotImplementedError("`one_int=False` is not on the accelerated path")
    is_np = isinstance(Wx, np.ndarray)
    W = torch.as_tensor(Wx)
    if not W.is_complex():
        raise ValueError("`Wx` must be complex")
    L.require_cuda()
    grad = A.needs_grad(W)
    if grad and rpadded:
        raise NotImplementedError("gradients of icwt with rpadded=True are not "
                                  "implemented")
    W = W.to(_device_of(Wx)).contiguous()
    is3 = W.ndim == 3
    W3 = W if is3 else W[None]
    B, na, n = W3.shape
    x_len = x_len or n
    if not isinstance(scales, (np.ndarray, torch.Tensor)) and nv is None:
        nv = 32
    wavelet = P.process_gmw_wavelet(wavelet, l1_norm)
    wavelet = P.Wavelet._init_if_not_isinstance(wavelet)
    ip = _icwt_plan(wavelet, scales, x_len, nv, l1_norm)
    if len(ip['weights']) != na:
        raise AssertionError("%s != %s" % (len(ip['weights']), na))
    xm = np.broadcast_to(np.asarray(x_mean, np.float64).ravel(), (B,)) \
        if np.size(x_mean) in (1, B) else None
    if xm is None:
        raise ValueError("`x_mean` must be a scalar or have one value per input")
    prec = L.F64 if W3.dtype == torch.complex128 else L.F32
    wd = _on_device(ip, 'weights', W3.device)

    def run(Win):
        Win = Win.contiguous()
        out = torch.empty((B, n), dtype=torch.float64 if prec else torch.float32,
                          device=Win.device)
        xmd = _dev_f64(xm, Win.device)
        with torch.cuda.device(Win.device):
            rc = L.load().ssqb_icwt(L.ptr(Win), L.ptr(wd), L.ptr(xmd),
                                    float(ip['mean_mult']), B, na, n, prec, L.ptr(out),
                                    L.stream_ptr())
        L.check(rc, 'icwt')
        return out, wd

    if grad:
        out = A.IcwtFn.apply(W3, run)
    else:
        out, _ = run(W3)
    out = out if is3 else out[0]
    return out.cpu().numpy() if is_np else out


def _icwt_plan(wavelet, scales, x_len, nv, l1_norm):
    """Row weights of the one-integral inverse (cached float64)."""
    def make():
        if isinstance(scales, str):
            sc, st, _, nv_ = P.process_scales(scales, x_len, wavelet, nv=nv,
                                              get_params=True)
        else:
            sc, st, _, nv_ = P.process_scales(P._to_numpy(scales), x_len,
                                              get_params=True)
        # the transition of log-piecewise scales is found at the caller's
        # dtype (float32 tolerances for float32 scales, cwt_utils.py:385)
        idx = (P.logscale_transition_idx(np.asarray(sc).ravel())
               if st == 'log-piecewise' else None)
        sc = np.asarray(sc, np.float64).ravel()
        weights, mean_mult = _icwt_weights(sc, st, P.adm_ssq(wavelet), l1_norm, idx)
        return dict(weights=weights, mean_mult=mean_mult)
    return _plan(('icwt', _wkey(wavelet), x_len, _akey(scales), nv, l1_norm), make)


def _icwt_weights(scales, scaletype, Cpsi, l1_norm, idx=None):
    """Per-row weights and the x_mean multiplicity of the one-integral inverse
    (_cwt.py:422-452, 479-494); `idx` the log-piecewise transition when known."""
    if scaletype == 'log-piecewise':
        idx = P.logscale_transition_idx(scales) if idx is None else idx
        if idx is None:
            raise ValueError("log-piecewise scales without a transition index")
        w0, _ = _icwt_weights(scales[:idx], 'log', Cpsi, l1_norm)
        w1, _ = _icwt_weights(scales[idx:], 'log', Cpsi, l1_norm)
        return np.concatenate([w0, w1]), 2.0  # each piece adds x_mean
    if scaletype == 'log':
        nv = int(np.round(1 / np.diff(np.log2(scales))[0]))
        norm = np.ones_like(scales) if l1_norm else scales**.5
        c = (2 / Cpsi) * np.log(2 ** (1 / nv))
    else:
        norm = scales if l1_norm else scales**1.5
        c = (2 / Cpsi) * np.pi / 4
    return c / norm, 1.0


#### inverse synchrosqueezing #################################################
def issq_cwt(Tx, wavelet='gmw', cc=None, cw=None):
    """Inverse synchrosqueezed CWT (_ssq_cwt.py:313-363): x = (2/Css) sum_k
    Re Tx[k]; with curve centres `cc` and widths `cw` (N, K), the K
    components over their row bands and the remainder, (K + 1, N) float64.
    Same container kind as `Tx`."""
    wavelet = P.Wavelet._init_if_not_isinstance(wavelet)
    return _issq(Tx, cc, cw, 2 / P.adm_ssq(wavelet))


def issq_stft(Tx, window=None, cc=None, cw=None, n_fft=None, win_len=None,
              hop_len=1, modulated=True):
    """Inverse synchrosqueezed STFT (_ssq_stft.py:139-198): as `issq_cwt`
    with the scale 2 / window[n_fft // 2]."""
    if not modulated:
        raise ValueError("inversion with `modulated == False` is unsupported.")
    if hop_len != 1:
        raise ValueError("inversion with `hop_len != 1` is unsupported.")
    n_fft = n_fft or (Tx.shape[0] - 1) * 2
    win_len = win_len or n_fft
    window, _ = P.get_window(window, win_len, n_fft=n_fft)
    _check_nola(window, hop_len)
    if abs(np.argmax(window) - len(window) // 2) > 1:
        warnings.warn("`window` maximum not centered; results may be inaccurate.")
    return _issq(Tx, cc, cw, 2 / window[len(window) // 2])


def _check_nola(window, hop_len):
    """Warnings of _stft.py:313-320 (non-zero overlap-add)."""
    from scipy import signal as sig
    if hop_len > len(window):
        warnings.warn("`hop_len > len(window)`; STFT not invertible")
    elif not sig.check_NOLA(window, len(window), len(window) - hop_len):
        warnings.warn("`window` fails Non-zero Overlap Add (NOLA) criterion; "
                      "STFT not invertible")


def _issq(Tx, cc, cw, scale):
    is_np = isinstance(Tx, np.ndarray)
    T = torch.as_tensor(Tx)
    if not T.is_complex():
        raise ValueError("`Tx` must be complex")
    if T.ndim != 2:
        raise ValueError("`Tx` must be 2D (rows, time) (got ndim=%s)" % T.ndim)
    L.require_cuda()
    dev = _device_of(Tx)
    T = T.to(dev).contiguous()
    nrows, N = T.shape
    prec = L.F64 if T.dtype == torch.complex128 else L.F32
    if cc is None and cw is None:
        K, ccd, cwd = 0, None, None
        out = torch.empty(N, dtype=torch.float64 if prec else torch.float32, device=dev)
    else:
        cc = np.asarray(P._to_numpy(cc))
        cw = np.asarray(P._to_numpy(cw))
        cc = (cc.reshape(-1, 1) if cc.ndim == 1 else cc).astype(np.int32)
        cw = (cw.reshape(-1, 1) if cw.ndim == 1 else cw).astype(np.int32)
        if cc.shape != cw.shape or cc.shape[0] != N:
            raise ValueError("`cc` and `cw` must both be (%d, K) (got %s, %s)"
                             % (N, cc.shape, cw.shape))
        K = cc.shape[1]
        ccd = torch.as_tensor(np.ascontiguousarray(cc), device=dev)
        cwd = torch.as_tensor(np.ascontiguousarray(cw), device=dev)
        out = torch.empty((K + 1, N), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        rc = L.load().ssqb_issq(L.ptr(T), nrows, N, L.ptr(ccd), L.ptr(cwd), K,
                                float(scale), prec, L.ptr(out), L.stream_ptr())
    L.check(rc, 'issq')
    return out.cpu().numpy() if is_np else out


#### squeeze on existing transforms ##########################################
def ssqueeze(Wx, w=None, ssq_freqs=None, scales=None, Sfs=None, fs=None, t=None,
             squeezing='sum', maprange='maximal', wavelet=None, gamma=None,
             was_padded=True, flipud=False, dWx=None, transform='cwt'):
    """Synchrosqueeze an existing CWT / STFT (ssqueezing.py:13-224). Returns
    `(Tx, ssq_freqs)` with Tx as a CUDA tensor."""
    if transform not in ('cwt', 'stft'):
        raise ValueError("`transform` must be one of: cwt, stft "
                         "(got %s)" % transform)
    if w is None and (dWx is None or gamma is None):
        raise ValueError("if `w` is None, `dWx` and `gamma` must not be.")
    _check_ssq_args(squeezing, maprange, 'trig')
    if transform == 'cwt' and scales is None:
        raise ValueError("`scales` can't be None if `transform == 'cwt'`")
    L.require_cuda()
    dev = _device_of(Wx)
    W = torch.as_tensor(Wx).to(dev).contiguous()
    W3 = W if W.ndim == 3 else W[None]
    B, na, N = W3.shape
    if w is not None:
        wt = torch.as_tensor(w).to(dev).contiguous()
        if float(wt.min()) < 0:
            raise ValueError("found negatives in `w`")
    dt, *_ = P.process_fs_and_t(fs, t, N)
    if transform == 'cwt':
        sc, cwt_st, _, nv = P.process_scales(P._to_numpy(scales), N,
                                             get_params=True)
        if isinstance(ssq_freqs, (np.ndarray, torch.Tensor)):
            f = P._to_numpy(ssq_freqs).astype(np.float64).ravel()
            logscale = P.infer_scaletype(f)[0].startswith('log')
        else:
            st = ssq_freqs if isinstance(ssq_freqs, str) else cwt_st
            if ((maprange == 'maximal' or isinstance(maprange, tuple)) and
                    st == 'log-piecewise'):
                raise ValueError("can't have `ssq_scaletype = log-piecewise` or "
                                 "tuple with `maprange = 'maximal'`")
            wav = P.Wavelet._init_if_not_isinstance(wavelet) if wavelet else None
            if wav is None and maprange != 'maximal' and \
                    not isinstance(maprange, tuple):
                raise ValueError(f"maprange='{maprange}' requires `wavelet`")
            f = P.compute_associated_frequencies(sc, N, wav, st, maprange,
                                                 was_padded, dt, 'cwt')
            logscale = st.startswith('log')
        const = P.squeeze_weights(sc, cwt_st, nv, 'cwt')
        sfs = None
    else:
        f = P._to_numpy(ssq_freqs).astype(np.float64).ravel()
        logscale = False
        const = P.squeeze_weights(None, None, None, 'stft', ssq_freqs=f)
        sfs = _dev_f64(P._to_numpy(Sfs), dev) if Sfs is not None else None
    mode, bp = P.bin_params(f, logscale)
    cst = _dev_f64(const, dev)
    Wv = _squeeze_values(W, squeezing)
    Wv = Wv if W.ndim == 3 else Wv[None]
    dW = None
    if w is None:
        dW = torch.as_tensor(dWx).to(dev).contiguous()
        dW = dW if dW.ndim == 3 else dW[None]
    Tx = _squeeze_from(Wv, wt if w is not None else None, dW, sfs, cst, mode, bp, na,
                       flipud, gamma if gamma is not None else 0.)
    Tx = Tx if W.ndim == 3 else Tx[0]
    if (transform == 'cwt' and not flipud) or flipud:
        f = f[::-1]
    return Tx, f


def phase_cwt(Wx, dWx, difftype='trig', gamma=None):
    """Phase transform of a CWT, inf where |Wx| < gamma (default sqrt(eps)
    of the data type), _ssq_cwt.py:420-509: |Im(dWx / Wx)| / 2pi for
    difftype 'trig'; for 'phase' the steps of the angle of Wx unwrapped along
    time (`dWx` unused), the last column the whole unwrapped excursion."""
    if difftype not in ('trig', 'phase'):
        raise ValueError(f"unsupported `difftype` '{difftype}'; must be one of "
                         "'trig', 'phase'.")
    W = torch.as_tensor(Wx)
    if gamma is None:
        gamma = np.sqrt(P.EPS64 if W.dtype == torch.complex128 else P.EPS32)
    if difftype == 'phase':
        return _phase_diff(W, 1, 4, 1., gamma)
    dW = torch.as_tensor(dWx)
    return _phase(W, dW, None, gamma)


def phase_cwt_num(Wx, dt, difforder=4, gamma=None):
    """Phase transform from numeric differences of Wx along time, periodic
    over the row (phase_cwt_num, _ssq_cwt.py:512-586): |Im(D Wx / Wx)| / 2pi,
    D of order 1, 2 or 4; inf where |Wx| < gamma (default 10 eps)."""
    if difforder not in (1, 2, 4):
        raise ValueError("`difforder` must be one of: 1, 2, 4 "
                         "(got %s)" % difforder)
    W = torch.as_tensor(Wx)
    gamma = gamma or _default_gamma('float64' if W.dtype == torch.complex128 else
                                    'float32')
    return _phase_diff(W, 2, difforder, dt, gamma)


def _phase_diff(W, mode, difforder, dt, gamma):
    if not W.is_complex():
        raise ValueError("`Wx` must be complex")
    L.require_cuda()
    dev = _device_of(W)
    W3 = W.to(dev).contiguous()
    W3 = W3 if W3.ndim == 3 else W3[None]
    B, na, N = W3.shape
    prec = L.F64 if W3.dtype == torch.complex128 else L.F32
    w = torch.empty((B, na, N), dtype=W3.real.dtype, device=dev)
    with torch.cuda.device(dev):
        rc = L.load().ssqb_phase_diff(L.ptr(W3), B, na, N, 0, N, mode, int(difforder),
                                      float(dt), float(gamma), prec, L.ptr(w),
                                      L.stream_ptr())
    L.check(rc, 'phase_diff')
    return w if W.ndim == 3 else w[0]


def phase_stft(Sx, dSx, Sfs, gamma=None):
    """|Sfs - Im(dSx / Sx) / 2pi|, inf where |Sx| < gamma
    (_ssq_stft.py:201-246)."""
    S = torch.as_tensor(Sx)
    gamma = _default_gamma('float64' if S.dtype == torch.complex128 else
                           'float32') if gamma is None else gamma
    return _phase(S, torch.as_tensor(dSx), Sfs, gamma)


def _phase(W, dW, Sfs, gamma):
    # an indexed_sum-free phase transform: reuse the squeeze's phase math by
    # running the STFT/CWT phase kernel path through ssqueeze_fast is not
    # possible (it sums); compute with the same float64 formula on the device
    L.require_cuda()
    dev = _device_of(W)
    W = W.to(dev)
    dW = dW.to(dev)
    c, d = W.real.double(), W.imag.double()
    a, b = dW.real.double(), dW.imag.double()
    ph = (b * c - a * d) / ((c * c + d * d) * 6.283185307179586)
    if Sfs is not None:
        s = torch.as_tensor(P._to_numpy(Sfs), dtype=torch.float64, device=dev)
        ph = s.reshape(-1, 1) - ph
    w = ph.abs()
    w = torch.where(W.abs() < gamma, torch.full_like(w, float('inf')), w)
    return w.to(W.real.dtype)


#### STFT ####################################################################
def _stft_core(x, window, n_fft, win_len, hop_len, fs, t, padtype, modulated,
               derivative, dtype, want_idx=False, want_w=False, bins=None,
               gamma=None, flipud=False):
    N = x.shape[-1]
    _, fs, _ = P.process_fs_and_t(fs, t, N)
    n_fft = n_fft or min(N // hop_len, 512)
    if win_len is None:
        win_len = (len(window) if isinstance(window, (np.ndarray, torch.Tensor))
                   else n_fft)
    dtype = P._dtype_str(dtype or P.DEFAULTS['stft_dtype'])
    win, dwin = P.get_window(window, win_len, n_fft, derivative=True)
    if (n_fft & (n_fft - 1) == 0 and not 8 <= n_fft <= 4096) or \
            (n_fft & (n_fft - 1) and not 4 <= n_fft <= 1024):
        raise NotImplementedError("n_fft must be a power of two in [8, 4096] or any "
                                  "length in [4, 1024] on the accelerated path "
                                  "(got %s)" % n_fft)
    if len(win) != n_fft:
        raise ValueError("window length %s != n_fft %s" % (len(win), n_fft))
    if padtype not in L.PADTYPES:
        raise ValueError("`padtype` must be one of %s" % list(L.PADTYPES))
    xd, is_2d = _to_device(x, dtype, False)
    dev = xd.device
    B = xd.shape[0]
    _, n1, _ = P.pad_geometry(N, N + n_fft - 1)
    nrow = n_fft // 2 + 1
    nframes = (N - 1) // hop_len + 1
    Sfs = np.linspace(0, .5 * fs, nrow)
    cdt, rdt = _CDT[dtype], _RDT[dtype]
    Sx = torch.empty((B, nrow, nframes), dtype=cdt, device=dev)
    dSx = torch.empty_like(Sx) if derivative else None
    w = torch.empty((B, nrow, nframes), dtype=rdt, device=dev) if want_w else None
    ipitch = L.idx_pitch(nframes)
    idx = (torch.empty((B, nrow, ipitch), dtype=torch.uint16, device=dev)
           if want_idx else None)
    dwin_s = dwin * fs if modulated else dwin  # _stft.py:132-135
    wd, dwd, sfd = _dev_f64(win, dev), _dev_f64(dwin_s, dev), _dev_f64(Sfs, dev)
    cb = None
    if bins is not None:
        cb = L.make_bins(bins[0], bins[1], nrow, flipud)
    gamma = _default_gamma(dtype) if gamma is None else gamma
    with torch.cuda.device(dev):
        rc = L.load().ssqb_stft(L.ptr(xd), B, N, n_fft, hop_len, n1,
                                L.PADTYPES[padtype], 1 if modulated else 0,
                                L.ptr(wd), L.ptr(dwd), L.ptr(sfd), cb, float(gamma),
                                _prec(dtype), L.ptr(Sx), L.ptr(dSx), L.ptr(w),
                                L.ptr(idx), ipitch, L.stream_ptr())
    L.check(rc, 'stft')
    return dict(Sx=Sx, dSx=dSx, w=w, idx=idx, ipitch=ipitch, Sfs=Sfs, dtype=dtype,
                dev=dev, is_2d=is_2d, B=B, nrow=nrow, nframes=nframes, fs=fs, gamma=gamma,
                N=N, n_fft=n_fft, hop=hop_len, n1=n1, ptype=L.PADTYPES[padtype],
                modulated=modulated, wd=wd, prec=_prec(dtype))


def stft(x, window=None, n_fft=None, win_len=None, hop_len=1, fs=None, t=None,
         padtype='reflect', modulated=True, derivative=False, dtype=None):
    """Short-Time Fourier Transform; returns `Sx` or `(Sx, dSx)`, CUDA tensors
    of shape (n_fft//2 + 1, n_frames) (_stft.py:13-181)."""
    def run(xin):
        return _stft_core(xin, window, n_fft, win_len, hop_len, fs, t, padtype, modulated,
                          derivative, dtype)
    if A.needs_grad(x):
        _grad_checks(True, False, padtype)
        holder = {}

        def run_keep(xin):
            holder['r'] = run(xin)
            return holder['r']
        outs = A.StftFn.apply(x, run_keep)
        r = holder['r']
        S, dS = outs if derivative else (outs, None)
    else:
        r = run(x)
        S, dS = r['Sx'], r['dSx']
    Sx, dSx = _out(S, True, r['is_2d']), _out(dS, True, r['is_2d'])
    return (Sx, dSx) if derivative else Sx


def trigdiff(A, fs=1., padtype=None, rpadded=None, N=None, n1=None, window=None,
             transform='cwt'):
    """Frequency-domain derivative of the rows of `A` (trigdiff,
    utils/common.py:161-245): ifft(fft(A) * 1j * xi * fs) along the last axis,
    A padded first unless `rpadded` (padtype defaults to 'reflect' then), and
    the result cut to columns n1 .. n1 + N of the padded length (N defaults to
    the padded length and the cut stops at its end, as in the reference).
    On the GPU (`ssqb_trigdiff`); numpy in, numpy out."""
    if transform == 'stft':
        raise NotImplementedError("`transform='stft'` is currently not supported.")
    is_np = isinstance(A, np.ndarray)
    T = torch.as_tensor(A)
    if T.ndim not in (2, 3):
        raise AssertionError("`A` must be 2D or 3D (got %s dims)" % T.ndim)
    if rpadded and N is None:
        raise ValueError("must pass `N` if `rpadded`")
    rpadded = rpadded or False
    padtype = padtype or ('reflect' if not rpadded else None)
    M = T.shape[-1]
    if padtype is not None:
        # padsignal (utils/common.py:54-158): 1D / 2D only; tensors 'zero' or
        # 'reflect', numpy arrays all five modes
        supported = ('zero', 'reflect', 'symmetric', 'replicate', 'wrap') if is_np else \
            ('zero', 'reflect')
        if padtype not in supported:
            raise ValueError("`padtype` must be one of: %s (got %s)"
                             % (', '.join(supported), padtype))
        if T.ndim != 2:
            raise ValueError("`x` must be 1D or 2D (got x.ndim == %s)" % T.ndim)
        Npad, n1, _ = P.p2up(M)  # the padding's n1 replaces the argument's
        ptype = L.PADTYPES[padtype]
    else:
        Npad, ptype = M, 5
        if Npad & (Npad - 1) or Npad < 8 or Npad > (1 << 22):
            raise NotImplementedError("trigdiff of an unpadded length needs a power of "
                                      "two in [8, 2^22] on the accelerated path")
        if n1 is None:
            _, n1, _ = P.p2up(N)
    Nn = N if N is not None else Npad
    N_out = min(Nn, Npad - n1)
    if N_out < 1:
        raise ValueError("empty output: n1=%s, N=%s, padded length %s" % (n1, Nn, Npad))
    L.require_cuda()
    dev = _device_of(A)
    cdt = torch.complex128 if T.dtype in (torch.complex128, torch.float64) else \
        torch.complex64
    T = T.to(device=dev, dtype=cdt).contiguous()
    rows = T.numel() // M
    out = torch.empty(T.shape[:-1] + (N_out,), dtype=cdt, device=dev)
    lib = L.load()
    wsb = lib.ssqb_trigdiff_workspace_bytes(rows, Npad)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    prec = L.F64 if cdt == torch.complex128 else L.F32
    with torch.cuda.device(dev):
        pad_n1 = n1 if padtype is not None else 0   # left pad of the input
        rc = lib.ssqb_trigdiff(L.ptr(T), rows, M, Npad, int(pad_n1), ptype, float(fs),
                               int(n1), int(N_out), prec, L.ptr(out), L.ptr(ws), wsb,
                               L.stream_ptr())
    L.check(rc, 'trigdiff')
    return out.cpu().numpy() if is_np else out


def _istft_plan(window, win_len, n_fft, hop_len, win_exp, dtype):
    """Window powers of the inverse STFT and the NOLA checks' warnings
    (_stft.py:230-237, 313-337), cached. The window is rounded to the data
    type first and its powers taken there, as the reference does."""
    def make():
        from scipy import signal as sig
        win, _ = P.get_window(window, win_len, n_fft)
        win = win.astype(dtype)
        msgs = []
        if hop_len > len(win):
            msgs.append("`hop_len > len(window)`; STFT not invertible")
        elif not sig.check_NOLA(win, len(win), len(win) - hop_len):
            msgs.append("`window` fails Non-zero Overlap Add (NOLA) criterion; "
                        "STFT not invertible")
        if dtype == 'float32' and not sig.check_NOLA(win, len(win), len(win) - hop_len,
                                                     tol=1e-3):
            msgs.append("Imprecision expected at right-most hop of signal, in "
                        "inversion. Lower `hop_len`, choose wider `window`, or use "
                        "`dtype='float64'`.")
        wa = np.ones_like(win) if win_exp == 0 else (win if win_exp == 1 else
                                                      win ** win_exp)
        w1 = win ** (win_exp + 1)
        return dict(wa=np.asarray(wa, np.float64), w1=np.asarray(w1, np.float64),
                    msgs=msgs)
    return _plan(('istft', _akey(window), win_len, n_fft, hop_len, win_exp, dtype), make)


def istft(Sx, window=None, n_fft=None, win_len=None, hop_len=1, N=None,
          modulated=True, win_exp=1):
    """Inverse STFT (_stft.py:184-256): per frame an inverse real FFT
    (fftshifted when `modulated`), overlap-added with window^win_exp and
    divided by the window norm sum of window^(win_exp+1), on the GPU. `Sx`
    (n_fft//2+1, n_frames), or batched (B, n_fft//2+1, n_frames); returns
    (N,) or (B, N), a numpy array for a numpy `Sx`, else a CUDA tensor."""
    is_np = isinstance(Sx, np.ndarray)
    S = torch.as_tensor(Sx)
    if not S.is_complex():
        raise ValueError("`Sx` must be complex")
    is3 = S.ndim == 3
    S3 = S if is3 else S[None]
    if S3.ndim != 3:
        raise ValueError("`Sx` must be 2D or 3D (got %s dims)" % S.ndim)
    B, nrow, nframes = S3.shape
    n_fft = n_fft or (nrow - 1) * 2
    win_len = win_len or n_fft
    N = N or hop_len * nframes
    dtype = 'float32' if S.dtype == torch.complex64 else 'float64'
    if (n_fft & (n_fft - 1) == 0 and not 8 <= n_fft <= 4096) or \
            (n_fft & (n_fft - 1) and not 4 <= n_fft <= 1024):
        raise NotImplementedError("n_fft must be a power of two in [8, 4096] or any "
                                  "length in [4, 1024] on the accelerated path "
                                  "(got %s)" % n_fft)
    if nrow != n_fft // 2 + 1:
        raise NotImplementedError("`Sx` must have n_fft//2 + 1 rows on the "
                                  "accelerated path (got %s for n_fft=%s)" % (nrow, n_fft))
    if (nframes - 1) * hop_len > N - 1:
        raise ValueError("%s frames at hop_len=%s end past a signal of N=%s"
                         % (nframes, hop_len, N))
    ip = _istft_plan(window, win_len, n_fft, hop_len, win_exp, dtype)
    for m in ip['msgs']:
        warnings.warn(m)
    L.require_cuda()
    dev = _device_of(Sx)
    S3 = S3.to(dev).contiguous()
    wa, w1 = _on_device(ip, 'wa', dev), _on_device(ip, 'w1', dev)
    prec = _prec(dtype)
    x = torch.empty((B, N), dtype=_RDT[dtype], device=dev)
    lib = L.load()
    wsb = lib.ssqb_istft_workspace_bytes(B, n_fft, nframes, prec)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        rc = lib.ssqb_istft(L.ptr(S3), B, n_fft, nframes, hop_len, N,
                            1 if modulated else 0, L.ptr(wa), L.ptr(w1),
                            float(np.finfo(dtype).tiny), prec, L.ptr(x), L.ptr(ws), wsb,
                            L.stream_ptr())
    L.check(rc, 'istft')
    x = x if is3 else x[0]
    return x.cpu().numpy() if is_np else x


def ssq_stft(x, window=None, n_fft=None, win_len=None, hop_len=1, fs=None, t=None,
             modulated=True, ssq_freqs=None, padtype='reflect', squeezing='sum',
             gamma=None, preserve_transform=None, dtype=None, astensor=True,
             flipud=False, get_w=False, get_dWx=False):
    """Synchrosqueezed STFT; returns `(Tx, Sx, ssq_freqs, Sfs[, w][, dSx])`
    (_ssq_stft.py:13-136)."""
    if x.ndim == 2 and get_w:
        raise NotImplementedError("`get_w=True` unsupported with batched input.")
    _check_ssq_args(squeezing, 'maximal', 'trig')
    if isinstance(ssq_freqs, np.ndarray) and P.infer_scaletype(ssq_freqs)[0] != 'linear':
        raise ValueError("`ssq_freqs` must be linearly distributed for `ssq_stft`")
    N = x.shape[-1]
    _, fs_, _ = P.process_fs_and_t(fs, t, N)
    nfft_ = n_fft or min(N // hop_len, 512)
    nrow = nfft_ // 2 + 1
    Sfs_np = np.linspace(0, .5 * fs_, nrow)
    f = Sfs_np if ssq_freqs is None else P._to_numpy(ssq_freqs).astype(np.float64).ravel()
    mode, bp = P.bin_params(f, False)
    const = P.squeeze_weights(None, None, None, 'stft', ssq_freqs=f)

    plain = isinstance(squeezing, str) and squeezing == 'sum'

    def run(xin):
        if not plain:
            # the squeeze sums other values than Sx (ssqueezing.py:196-201)
            r = _stft_core(xin, window, n_fft, win_len, hop_len, fs, t, padtype, modulated,
                           True, dtype, want_w=get_w, gamma=gamma, flipud=flipud)
            is2 = r['is_2d']
            Sv = _squeeze_values(r['Sx'] if is2 else r['Sx'][0], squeezing)
            cst = _dev_f64(const, r['dev'])
            Tx = _squeeze_from(Sv if is2 else Sv[None], r['w'], r['dSx'],
                               _dev_f64(r['Sfs'], r['dev']), cst, mode, bp, r['nrow'],
                               flipud, r['gamma'])
            return Tx, r, cst
        r = _stft_core(xin, window, n_fft, win_len, hop_len, fs, t, padtype, modulated,
                       get_dWx, dtype, want_idx=True, want_w=get_w, bins=(mode, bp),
                       gamma=gamma, flipud=flipud)
        Tx = torch.empty_like(r['Sx'])
        cst = _dev_f64(const, r['dev'])
        with torch.cuda.device(r['dev']):
            rc = L.load().ssqb_squeeze(L.ptr(r['Sx']), L.ptr(r['idx']), r['ipitch'],
                                       L.ptr(cst), r['B'], r['nrow'], r['nframes'],
                                       r['nrow'], _prec(r['dtype']), L.ptr(Tx),
                                       L.stream_ptr())
        L.check(rc, 'squeeze')
        return Tx, r, cst

    if A.needs_grad(x):
        _grad_checks(astensor, False, padtype)
        if not plain:
            raise NotImplementedError("gradients need squeezing='sum'")
        holder = {}

        def run_keep(xin):
            holder['out'] = run(xin)
            return holder['out']
        Tx, Sx = A.SsqStftFn.apply(x, run_keep)
        r = holder['out'][1]
    else:
        Tx, r, _ = run(x)
        Sx = r['Sx']
    is2 = r['is_2d']
    Sfs_out = Sfs_np.astype(r['dtype'])
    f_out = f.astype(r['dtype']) if ssq_freqs is None else f
    if flipud:
        f_out = f_out[::-1]
    if astensor:
        Sfs_out = torch.as_tensor(Sfs_out, device=r['dev'])
        f_out = torch.as_tensor(np.ascontiguousarray(f_out), device=r['dev'])
    out = [_out(Tx, astensor, is2), _out(Sx, astensor, is2), f_out, Sfs_out]
    if get_w:
        out.append(_out(r['w'], astensor, is2))
    if get_dWx:
        out.append(_out(r['dSx'], astensor, is2))
    return tuple(out)
