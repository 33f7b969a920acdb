# -*- coding: utf-8 -*-
"""Reverse-mode differentiation of `cwt`, `ssq_cwt` and `icwt`.

ssqueezepy has no backward pass of its own (its torch-based GPU `cwt`,
_cwt.py:250-311, is differentiable only through torch's generic FFT
autograd). Here each transform is a `torch.autograd.Function` whose backward
calls the adjoint kernels of libssqb.so:

* `cwt`: the transposed CWT (`ssqb_cwt_adjoint`): per scale a forward FFT of
  the gradient, times the wavelet, summed over scales, one inverse FFT and
  the transpose of the padding.
* `ssq_cwt`: the squeeze's adjoint is a gather through the forward's bin
  index (bins held fixed: they are piecewise constant in x), fused into the
  row loader of the transposed CWT; the backward keeps only the uint16 bin
  index of the forward, never Wx.
* `icwt`: each row receives its weight times the output gradient
  (`ssqb_icwt_adjoint`).
* `stft` / `ssq_stft`: the transposed STFT (`ssqb_stft_adjoint`): per frame
  the real part of the inverse transform of the one-sided gradient, times
  the window, added back at the frame's samples, then the transpose of the
  padding; `ssq_stft`'s squeeze gather is fused into its loader.

Gradients of float32 transforms are computed in float32 arithmetic.
"""
import torch

from . import _lib as L


def needs_grad(*ts):
    return torch.is_grad_enabled() and any(
        isinstance(t, torch.Tensor) and t.requires_grad for t in ts)


def cwt_adjoint(r, gWx=None, gTx=None, sq_weights=None, gxr=None, icwt_weights=None):
    """Gradient of x (B, N) from the gradients of Wx / Tx / the icwt output
    of the forward described by `r` (the dict of `_cwt_core`)."""
    B, N, na = r['B'], r['N'], r['na']
    dev = r['dev']
    rdt = torch.float64 if r['prec'] == L.F64 else torch.float32
    cdt = torch.complex128 if r['prec'] == L.F64 else torch.complex64
    gx = torch.empty((B, N), dtype=rdt, device=dev)
    if gWx is None and gTx is None and gxr is None:
        return gx.zero_()
    lib = L.load()
    wsb = lib.ssqb_cwt_adjoint_workspace_bytes(B, r['Npad'], na, r['prec'])
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    gWx = None if gWx is None else gWx.to(cdt).reshape(B, na, N).contiguous()
    gTx = None if gTx is None else gTx.to(cdt).reshape(B, na, N).contiguous()
    gxr = None if gxr is None else gxr.to(rdt).reshape(B, N).contiguous()
    with torch.cuda.device(dev):
        rc = lib.ssqb_cwt_adjoint(
            L.ptr(gWx), L.ptr(gTx), L.ptr(r['idx'] if gTx is not None else None),
            r['ipitch'], L.ptr(sq_weights if gTx is not None else None), na, L.ptr(gxr),
            L.ptr(icwt_weights if gxr is not None else None), B, N, r['Npad'], r['n1'],
            r['ptype'], L.ptr(r['sc_d']), na, r['cw'], r['prec'], L.ptr(gx), 0, L.ptr(ws),
            wsb, L.stream_ptr())
    L.check(rc, 'cwt_adjoint')
    return gx


def _keep(r):
    """What the backward needs of a forward: geometry, scales, bin index;
    never the transform itself."""
    return {k: v for k, v in r.items() if k not in ('Wx', 'dWx', 'w')}


class CwtFn(torch.autograd.Function):
    """x -> Wx (and a non-differentiable dWx when the forward returns it)."""

    @staticmethod
    def forward(ctx, x, run):
        r = run(x)
        ctx.r = _keep(r)
        ctx.x_meta = (x.shape, x.dtype)
        if r['dWx'] is not None:
            ctx.mark_non_differentiable(r['dWx'])
            return r['Wx'], r['dWx']
        return r['Wx']

    @staticmethod
    def backward(ctx, gWx, *rest):
        gx = cwt_adjoint(ctx.r, gWx=gWx)
        shape, dtype = ctx.x_meta
        return gx.reshape(shape).to(dtype), None


class SsqCwtFn(torch.autograd.Function):
    """x -> (Tx, Wx); the backward needs only the forward's bin index."""

    @staticmethod
    def forward(ctx, x, run):
        Tx, r, cst = run(x)
        ctx.r, ctx.cst = _keep(r), cst
        ctx.x_meta = (x.shape, x.dtype)
        return Tx, r['Wx']

    @staticmethod
    def backward(ctx, gTx, gWx):
        gx = cwt_adjoint(ctx.r, gWx=gWx, gTx=gTx, sq_weights=ctx.cst)
        shape, dtype = ctx.x_meta
        return gx.reshape(shape).to(dtype), None


def stft_adjoint(r, gSx=None, gTx=None, sq_weights=None):
    """Gradient of x (B, N) from the gradients of Sx / Tx of the STFT forward
    described by `r` (the dict of `_stft_core`)."""
    B, N, nrow, nf = r['B'], r['N'], r['nrow'], r['nframes']
    dev = r['dev']
    rdt = torch.float64 if r['prec'] == L.F64 else torch.float32
    cdt = torch.complex128 if r['prec'] == L.F64 else torch.complex64
    gx = torch.empty((B, N), dtype=rdt, device=dev)
    if gSx is None and gTx is None:
        return gx.zero_()
    lib = L.load()
    wsb = lib.ssqb_stft_adjoint_workspace_bytes(B, N, r['n_fft'], r['hop'], r['prec'])
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    gSx = None if gSx is None else gSx.to(cdt).reshape(B, nrow, nf).contiguous()
    gTx = None if gTx is None else gTx.to(cdt).reshape(B, nrow, nf).contiguous()
    with torch.cuda.device(dev):
        rc = lib.ssqb_stft_adjoint(
            L.ptr(gSx), L.ptr(gTx), L.ptr(r['idx'] if gTx is not None else None),
            r['ipitch'], L.ptr(sq_weights if gTx is not None else None), B, N, r['n_fft'],
            r['hop'], r['n1'], r['ptype'], 1 if r['modulated'] else 0, L.ptr(r['wd']),
            r['prec'], L.ptr(gx), 0, L.ptr(ws), wsb, L.stream_ptr())
    L.check(rc, 'stft_adjoint')
    return gx


def _keep_stft(r):
    return {k: v for k, v in r.items() if k not in ('Sx', 'dSx', 'w')}


class StftFn(torch.autograd.Function):
    """x -> Sx (and a non-differentiable dSx when the forward returns it)."""

    @staticmethod
    def forward(ctx, x, run):
        r = run(x)
        ctx.r = _keep_stft(r)
        ctx.x_meta = (x.shape, x.dtype)
        if r['dSx'] is not None:
            ctx.mark_non_differentiable(r['dSx'])
            return r['Sx'], r['dSx']
        return r['Sx']

    @staticmethod
    def backward(ctx, gSx, *rest):
        gx = stft_adjoint(ctx.r, gSx=gSx)
        shape, dtype = ctx.x_meta
        return gx.reshape(shape).to(dtype), None


class SsqStftFn(torch.autograd.Function):
    """x -> (Tx, Sx); the backward needs only the forward's bin index."""

    @staticmethod
    def forward(ctx, x, run):
        Tx, r, cst = run(x)
        ctx.r, ctx.cst = _keep_stft(r), cst
        ctx.x_meta = (x.shape, x.dtype)
        return Tx, r['Sx']

    @staticmethod
    def backward(ctx, gTx, gSx):
        gx = stft_adjoint(ctx.r, gSx=gSx, gTx=gTx, sq_weights=ctx.cst)
        shape, dtype = ctx.x_meta
        return gx.reshape(shape).to(dtype), None


class IcwtFn(torch.autograd.Function):
    """Wx (B, na, n) -> x (B, n)."""

    @staticmethod
    def forward(ctx, W3, run):
        out, weights = run(W3)
        ctx.weights = weights
        ctx.meta = (W3.shape, W3.dtype, W3.device)
        return out

    @staticmethod
    def backward(ctx, gx):
        shape, dtype, dev = ctx.meta
        B, na, n = shape
        prec = L.F64 if dtype == torch.complex128 else L.F32
        rdt = torch.float64 if prec == L.F64 else torch.float32
        gW = torch.empty(shape, dtype=dtype, device=dev)
        g = gx.to(rdt).reshape(B, n).contiguous()
        with torch.cuda.device(dev):
            rc = L.load().ssqb_icwt_adjoint(L.ptr(g), L.ptr(ctx.weights), B, na, n, prec,
                                            L.ptr(gW), 0, L.stream_ptr())
        L.check(rc, 'icwt_adjoint')
        return gW, None
