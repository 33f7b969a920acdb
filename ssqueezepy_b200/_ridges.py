# -*- coding: utf-8 -*-
"""`extract_ridges` on the GPU (ridge_extraction.py:11-232).

Same arguments and returns as ssqueezepy's: `ridge_idxs` (N, n_ridges) and,
with `get_params`, `ridge_f` (scales or frequencies along each ridge) and
`ridge_e` (energies). The arithmetic is the input's (float32 for complex64,
as the reference's `dtype`) and follows the reference's serial code path;
its `parallel=True` path updates the backward ridge from several threads at
once, so where two frequencies tie within eps it may keep either one, while
this one always keeps the highest, as the serial path does. `parallel` is
accepted for the signature and has no effect.
"""
import numpy as np
import torch

from . import _lib as L
from . import _params as P

__all__ = ['extract_ridges']


def extract_ridges(Tf, scales, penalty=2., n_ridges=1, bw=15, transform='cwt',
                   get_params=False, parallel=True):
    is_np = isinstance(Tf, np.ndarray)
    T = torch.as_tensor(Tf)
    if T.ndim != 2:
        raise ValueError("`Tf` must be a 2D array (frequencies, time)")
    if not T.is_complex():
        # real (or integer) input: the reference takes float32 eps, scales and
        # penalty for anything but complex128 (ridge_extraction.py:113-115);
        # here its energies are float32 too
        T = T.to(torch.complex64)
    if transform not in ('cwt', 'stft'):
        raise ValueError("`transform` must be 'cwt' or 'stft' (got %s)" % transform)
    L.require_cuda()
    dev = T.device if T.is_cuda else torch.device('cuda', torch.cuda.current_device())
    T = T.to(dev).contiguous()
    f64 = T.dtype == torch.complex128
    dt = np.float64 if f64 else np.float32
    eps = P.EPS64 if f64 else P.EPS32
    sc = np.asarray(P._to_numpy(scales), dt).squeeze()
    s = np.log(sc) if transform == 'cwt' else sc
    nf, N = T.shape
    if sc.shape != (nf,):
        raise ValueError("`scales` must have one value per row of `Tf` (%d)" % nf)
    tdt = torch.float64 if f64 else torch.float32
    s_d = torch.as_tensor(np.ascontiguousarray(s), dtype=tdt, device=dev)
    sc_d = torch.as_tensor(np.ascontiguousarray(sc), dtype=tdt, device=dev)
    idx = torch.empty((N, n_ridges), dtype=torch.int32, device=dev)
    rf = torch.empty((N, n_ridges), dtype=tdt, device=dev) if get_params else None
    re = torch.empty((N, n_ridges), dtype=tdt, device=dev) if get_params else None
    prec = L.F64 if f64 else L.F32
    lib = L.load()
    wsb = lib.ssqb_ridges_workspace_bytes(nf, N, prec)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        rc = lib.ssqb_extract_ridges(L.ptr(T), nf, N, L.ptr(s_d), L.ptr(sc_d),
                                     float(dt(penalty)), int(n_ridges), int(bw), float(eps),
                                     prec, L.ptr(idx), L.ptr(rf), L.ptr(re), L.ptr(ws), wsb,
                                     L.stream_ptr())
    L.check(rc, 'extract_ridges')
    if is_np:
        out = (idx.cpu().numpy().astype(int),) + ((rf.cpu().numpy(), re.cpu().numpy())
                                                  if get_params else ())
    else:
        out = (idx.long(),) + ((rf, re) if get_params else ())
    return out if get_params else out[0]
