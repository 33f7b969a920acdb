# -*- coding: utf-8 -*-
"""`ssq_cwt` over many float32 signals of uneven length in a few launches.

ssqueezepy transforms equal-length 2D input only (_cwt.py:270-271) and
squeezes it one signal at a time (ssqueezing.py:210-214); signals of
different lengths take one `ssq_cwt` call each. Here a plan
(`SsqCwtBatch`) packs the signals end to end, describes each by an
`ssqb_sig` (offsets, scales, squeeze weights, bin mapping), groups them by
padded length (`p2up`, utils/common.py:32-51) and runs, per group, one
`ssqb_cwt_batch` call (spectra + fused CWT with bin index) and then one
`ssqb_squeeze_batch` launch over all signals. The device work can be
captured once in a CUDA graph and replayed.

Per signal the results equal `ssq_cwt(x_i, ...)` of the same arguments:
`(Tx_i, Wx_i, ssq_freqs_i, scales_i)`.
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from . import _params as P
from . import _transforms as T

__all__ = ['SsqCwtBatch', 'ssq_cwt_batch', 'describe_signals']


def describe_signals(lengths, wavelet, scales='log-piecewise', nv=32, fs=None,
                     padtype='reflect', maprange='peak', flipud=True):
    """Host descriptors (`ssqb_sig` records, L.SIG_DTYPE) of signals packed end
    to end in the given order, with the float64 parameters of each signal's
    `ssq_cwt`. The `scales` / `weights` fields hold element offsets into the
    concatenated per-signal scale / weight arrays (the caller turns them into
    device pointers)."""
    wavelet = P.Wavelet._init_if_not_isinstance(wavelet)
    sig = np.zeros(len(lengths), L.SIG_DTYPE)
    d = dict(scales64=[], weights64=[], ssq_freqs=[], scales32=[], dt=None)
    xo = oo = io = so = 0
    for i, N in enumerate(lengths):
        N = int(N)
        dt, _, _ = P.process_fs_and_t(fs, None, N)
        if d['dt'] is None:
            d['dt'] = dt
        sp = T._scales_plan(scales, N, wavelet, nv)
        fp = T._ssq_plan(wavelet, scales, N, nv, None, maprange, padtype, dt, sp)
        na = sp['na']
        _, n1, _ = P.p2up(N)
        ip = L.idx_pitch(N)
        s = sig[i]
        s['x_off'], s['out_off'], s['idx_off'] = xo, oo, io
        s['N'], s['n1'], s['na'], s['idx_pitch'] = N, n1, na, ip
        bp = list(fp['bp'])
        s['mode'] = fp['mode']
        s['idx1'] = int(bp[4]) if len(bp) > 4 else 0
        s['flipud'] = 1 if flipud else 0
        s['nbins'] = na
        s['p'] = bp[:4]
        s['scales'] = s['weights'] = so
        d['scales64'].append(sp['scales'])
        d['weights64'].append(fp['const'])
        d['ssq_freqs'].append(fp['f_asc'][::-1])
        d['scales32'].append(sp['scales'].astype(np.float32))
        xo += N
        oo += na * N
        io += na * ip
        so += na
    d['n_x'], d['n_out'], d['n_idx'] = xo, oo, io
    return sig, d


class SsqCwtBatch:
    """Plan of `ssq_cwt` over float32 signals of the given lengths.

    Arguments follow `ssq_cwt` (wavelet, scales, nv, fs, padtype, maprange,
    flipud, gamma). Host parameters are computed once here; device buffers
    (packed input, Wx, Tx, bin index, workspace) belong to the plan, so each
    call overwrites the previous call's outputs. `graph=True` captures the
    device work in a CUDA graph after one eager run and replays it.
    `autotune=True` picks, per padded-length group, the intermediate budget
    (rows per tile and signals per chunk) and the band bound (which rows take
    the band-limited single pass) that run fastest on this device. Without
    it, rows whose wavelet band fits 512 bins take the band pass.
    """

    # intermediate budgets the autotuner tries per length group, bytes, and
    # band bounds (bins; -1 = no band pass)
    TUNE_BUDGETS = (64 << 20, 128 << 20, 256 << 20, 512 << 20)
    TUNE_BANDS = (-1, 256, 512, 1024)

    def __init__(self, lengths, wavelet='gmw', scales='log-piecewise', nv=32, fs=None,
                 padtype='reflect', maprange='peak', flipud=True, gamma=None,
                 device=None, graph=False, autotune=False):
        L.require_cuda()
        T._check_ssq_args('sum', maprange, 'trig')
        if padtype not in L.PADTYPES:
            raise ValueError("`padtype` must be one of %s (got %s)"
                             % (list(L.PADTYPES), padtype))
        self.lengths = [int(n) for n in lengths]
        if not self.lengths or min(self.lengths) < 4:
            raise ValueError("need at least one signal, each of length >= 4")
        self.dev = torch.device(device) if device is not None else \
            torch.device('cuda', torch.cuda.current_device())
        wavelet = P.Wavelet._init_if_not_isinstance(wavelet)
        if wavelet.dtype != 'float32':
            raise NotImplementedError("batches of uneven length take float32 "
                                      "wavelets (got %s)" % wavelet.dtype)
        self.wavelet = wavelet
        self.prec = T._prec('float32')
        self.ptype = L.PADTYPES[padtype]
        self.flipud = flipud
        self.gamma = T._default_gamma('float32') if gamma is None else float(gamma)
        sig, d = describe_signals(self.lengths, wavelet, scales, nv, fs, padtype,
                                  maprange, flipud)
        self.dt = d['dt']
        self.ssq_freqs, self.scales_np = d['ssq_freqs'], d['scales32']
        self.scales64, self.weights64 = d['scales64'], d['weights64']  # float64
        self.n_x, self.n_out, self.n_idx = d['n_x'], d['n_out'], d['n_idx']
        dev = self.dev
        self.scales_dev = torch.as_tensor(np.concatenate(self.scales64), device=dev)
        self.weights_dev = torch.as_tensor(np.concatenate(self.weights64), device=dev)
        soff = sig['scales'].copy()  # element offsets until here
        sig['scales'] = self.scales_dev.data_ptr() + 8 * soff
        sig['weights'] = self.weights_dev.data_ptr() + 8 * soff
        self.sig_np = sig

        # groups of one padded length; each keeps its own descriptor arrays
        npads = np.array([P.p2up(N)[0] for N in self.lengths])
        self.groups = []
        ws = 0
        lib = L.load()
        for Npad in sorted(set(npads.tolist())):
            sel = np.nonzero(npads == Npad)[0]
            hs = np.ascontiguousarray(sig[sel])
            self.groups.append(dict(Npad=int(Npad), n=len(sel), sel=sel, host=hs,
                                    dev=self._to_dev(hs)))
            ws = max(ws, lib.ssqb_cwt_batch_workspace_bytes(len(sel), int(Npad),
                                                            self.prec))
        self.sig_dev = self._to_dev(sig)
        self.cw = L.wavelet_struct(wavelet)
        for g in self.groups:  # the library's defaults per group
            g['ws'] = lib.ssqb_cwt_batch_workspace_bytes(g['n'], g['Npad'], self.prec)
            g['band'] = self._band(g, 0)
        if autotune:
            xb = max(g['n'] * g['Npad'] * 16 for g in self.groups)
            ws = max(ws, xb + max(self.TUNE_BUDGETS))
        self.ws_bytes = ws
        self.ws = torch.empty(ws, dtype=torch.uint8, device=dev)
        self.x = torch.empty(self.n_x, dtype=torch.float32, device=dev)
        self.Wx = torch.empty(self.n_out, dtype=torch.complex64, device=dev)
        self.Tx = torch.empty(self.n_out, dtype=torch.complex64, device=dev)
        self.idx = torch.empty(self.n_idx, dtype=torch.uint16, device=dev)
        self._host = torch.empty(self.n_x, dtype=torch.float32, pin_memory=True)
        self.use_graph = graph
        self._graph = None
        self._ran = False
        self.tuning = None
        if autotune:
            self.autotune()

    def _to_dev(self, arr):
        return torch.as_tensor(arr.view(np.uint8).copy(), device=self.dev)

    def _band(self, g, max_bins):
        """(band_from, band_log) of a length group: the rows from which every
        signal's wavelet bands fit 2^band_log <= max_bins bins (0: the
        library's default bound; -1: no band pass), from the host scales."""
        if max_bins < 0:
            return 1 << 30, 0
        lib = L.load()
        bf_all, bl_all = 0, 0
        bf, bl = ctypes.c_int(), ctypes.c_int()
        for i in g['sel']:
            sc = np.ascontiguousarray(self.scales64[i], np.float64)
            rc = lib.ssqb_cwt_band_rows(sc.ctypes.data, len(sc), g['Npad'], self.cw,
                                        self.prec, int(max_bins), ctypes.byref(bf),
                                        ctypes.byref(bl))
            L.check(rc, 'band_rows')
            bf_all, bl_all = max(bf_all, bf.value), max(bl_all, bl.value)
        na_max = int(max(len(self.scales64[i]) for i in g['sel']))
        return (bf_all, bl_all) if bf_all < na_max and bl_all >= 3 else (1 << 30, 0)

    @property
    def launches(self):
        """Kernel launches of one run (all groups plus the squeeze)."""
        lib = L.load()
        n = 1
        for g in self.groups:
            k = lib.ssqb_cwt_batch_ex_launches(g['host'].ctypes.data_as(ctypes.c_void_p),
                                               g['n'], g['Npad'], self.prec, g['ws'],
                                               *g['band'])
            if k < 0:
                raise RuntimeError("launch count query failed")
            n += k
        return n

    def _cwt_group(self, g, ws_bytes, st, band=None):
        lib = L.load()
        bf, bl = g['band'] if band is None else band
        rc = lib.ssqb_cwt_batch_ex(
            L.ptr(self.x), g['host'].ctypes.data_as(ctypes.c_void_p), L.ptr(g['dev']),
            g['n'], g['Npad'], self.ptype, self.cw, float(self.dt), self.gamma, self.prec,
            L.ptr(self.Wx), L.ptr(self.idx), L.ptr(self.ws), ws_bytes, bf, bl, st)
        L.check(rc, 'cwt_batch')

    def autotune(self, reps=2):
        """Per length group, time the CWT over a small search space and keep
        the fastest point: the intermediate budget (TUNE_BUDGETS: rows per
        tile and signals per chunk) times the band bound (TUNE_BANDS: the
        largest wavelet band, in bins, whose rows take the band-limited single
        pass instead of the tile passes; -1 = none), with CUDA events on the
        current stream. Runs on whatever is in the packed input (the values do
        not change the work)."""
        st = torch.cuda.current_stream(self.dev)
        sp = L.stream_ptr(st)
        if not self._ran:  # a seeded stand-in signal until the first load
            gen = torch.Generator(device=self.dev)
            gen.manual_seed(0)
            self.x.copy_(torch.randn(self.n_x, generator=gen, device=self.dev))
        self.tuning = []
        for g in self.groups:
            xb = g['n'] * g['Npad'] * 16
            times = {}
            bands = {mb: self._band(g, mb) for mb in self.TUNE_BANDS}
            for zb in self.TUNE_BUDGETS:
                wsb = min(self.ws_bytes, xb + zb)
                for mb, band in bands.items():
                    if mb >= 0 and band[0] >= (1 << 30):
                        continue  # no band rows at this bound
                    try:
                        self._cwt_group(g, wsb, sp, band)  # warm; small budgets refused
                    except RuntimeError:
                        continue
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    for _ in range(reps):
                        self._cwt_group(g, wsb, sp, band)
                    e1.record(st)
                    e1.synchronize()
                    times[(wsb, mb)] = e0.elapsed_time(e1) / reps
            (best_ws, best_mb) = min(times, key=times.get)
            g['ws'], g['band'] = best_ws, bands[best_mb]
            self.tuning.append(dict(
                Npad=g['Npad'], signals=g['n'], budget_mb=(best_ws - xb) / 2**20,
                band_bins=best_mb, band_from=bands[best_mb][0] if best_mb >= 0 else None,
                ms={'%d MB/%s' % (round((k[0] - xb) / 2**20),
                                  'off' if k[1] < 0 else ('%d bins' % k[1] if k[1] else
                                                          'default')): round(v, 3)
                    for k, v in times.items()}))
        self._graph = None
        return self.tuning

    def run(self):
        """The device work on the packed input `self.x` (graph replay once
        captured)."""
        if self._graph is not None:
            self._graph.replay()
            return
        if self.use_graph and self._ran:
            torch.cuda.synchronize(self.dev)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._enqueue()
            self._graph = g
            g.replay()
            return
        self._enqueue()
        self._ran = True

    def _enqueue(self):
        lib = L.load()
        st = L.stream_ptr()
        for g in self.groups:
            self._cwt_group(g, g['ws'], st)
        rc = lib.ssqb_squeeze_batch(
            L.ptr(self.Wx), L.ptr(self.idx), self.sig_np.ctypes.data_as(ctypes.c_void_p),
            L.ptr(self.sig_dev), len(self.lengths), self.prec, L.ptr(self.Tx), st)
        L.check(rc, 'squeeze_batch')

    def load(self, xs):
        """Copy the signals (sequence of 1D arrays / tensors) into the packed
        device input through pinned host memory."""
        if len(xs) != len(self.lengths):
            raise ValueError("expected %d signals, got %d" % (len(self.lengths), len(xs)))
        h = self._host.numpy()
        o = 0
        for x, N in zip(xs, self.lengths):
            if x.ndim != 1 or x.shape[-1] != N:
                raise ValueError("signal lengths must match the plan")
            if isinstance(x, torch.Tensor):
                x = x.detach().cpu().numpy()
            h[o:o + N] = x
            o += N
        self.x.copy_(self._host, non_blocking=True)

    def outputs(self):
        """Per signal `(Tx, Wx, ssq_freqs, scales)` views of the plan's
        buffers (ssq_freqs float64 numpy, high to low)."""
        out = []
        for i, s in enumerate(self.sig_np):
            na, N, o = int(s['na']), int(s['N']), int(s['out_off'])
            out.append((self.Tx[o:o + na * N].view(na, N),
                        self.Wx[o:o + na * N].view(na, N),
                        self.ssq_freqs[i],
                        torch.as_tensor(self.scales_np[i], device=self.dev)))
        return out

    def __call__(self, xs):
        self.load(xs)
        self.run()
        return self.outputs()


def ssq_cwt_batch(xs, wavelet='gmw', scales='log-piecewise', nv=32, fs=None,
                  padtype='reflect', maprange='peak', flipud=True, gamma=None):
    """`ssq_cwt` of each signal in `xs` (float32, any lengths), computed
    together; returns a list of `(Tx, Wx, ssq_freqs, scales)`. Builds a plan
    per call; reuse `SsqCwtBatch` to amortise host parameters and replay a
    CUDA graph."""
    plan = SsqCwtBatch([x.shape[-1] for x in xs], wavelet, scales, nv, fs, padtype,
                       maprange, flipud, gamma)
    return plan(xs)
