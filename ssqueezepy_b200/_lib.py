# -*- coding: utf-8 -*-
"""ctypes binding of the C ABI in include/ssqb.h (libssqb.so, built in-tree).

There is no CPU fallback: if the library or a CUDA device is missing, every
transform raises instead of computing something else.
"""
import ctypes
import os
import threading

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, '_lib', 'libssqb.so')

F32, F64, F32X = 0, 1, 2
OK, EINVAL, EUNSUPPORTED, ECUDA, EWORKSPACE = 0, 1, 2, 3, 4
NO_BIN = 0xFFFF
PADTYPES = {'zero': 0, 'reflect': 1, 'symmetric': 2, 'replicate': 3, 'wrap': 4}


class CWavelet(ctypes.Structure):
    _fields_ = [('kind', ctypes.c_int32), ('npoly', ctypes.c_int32),
                ('p', ctypes.c_double * 4), ('band', ctypes.c_double * 2),
                ('kc', ctypes.c_double * 8)]


class CBins(ctypes.Structure):
    _fields_ = [('mode', ctypes.c_int32), ('idx1', ctypes.c_int32),
                ('flipud', ctypes.c_int32), ('nbins', ctypes.c_int32),
                ('p', ctypes.c_double * 4)]


_vp, _i, _d, _sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
SIGNATURES = {
    'ssqb_version': (_i, []),
    'ssqb_last_error': (ctypes.c_char_p, []),
    'ssqb_device_status': (_i, [_vp, ctypes.POINTER(ctypes.c_int)]),
    'ssqb_cwt_workspace_bytes': (_sz, [_i, _i, _i, _i, _i]),
    'ssqb_cwt_launches': (_i, [_i, _i, _i, _i, _sz]),
    'ssqb_cwt': (_i, [_vp, _i, _i, _i, _i, _i, _i, _vp, _i,
                      ctypes.POINTER(CWavelet), _d, ctypes.POINTER(CBins), _d, _i,
                      _vp, _vp, _vp, _vp, _i, _vp, _sz, _vp]),
    'ssqb_cwt_ex': (_i, [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _i,
                         ctypes.POINTER(CWavelet), _d, ctypes.POINTER(CBins), _d, _i,
                         _vp, _vp, _vp, _vp, _i, _vp, _sz, _vp]),
    'ssqb_cwt_ex_launches': (_i, [_i, _i, _i, _i, _sz, _vp, ctypes.POINTER(CWavelet)]),
    'ssqb_squeeze': (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _i, _i, _vp, _vp]),
    'ssqb_ssqueeze_fast': (_i, [_vp, _vp, _vp, _vp, ctypes.POINTER(CBins), _d,
                                _i, _i, _i, _i, _vp, _vp]),
    'ssqb_indexed_sum': (_i, [_vp, _vp, _vp, ctypes.POINTER(CBins), _i, _i, _i,
                              _i, _vp, _vp]),
    'ssqb_stft': (_i, [_vp, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp,
                       ctypes.POINTER(CBins), _d, _i, _vp, _vp, _vp, _vp, _i, _vp]),
    'ssqb_icwt': (_i, [_vp, _vp, _vp, _d, _i, _i, _i, _i, _vp, _vp]),
    'ssqb_cwt_noalloc': (_i, [_vp, _i, _i, _i, _i, _i, _i, _vp, _i,
                              ctypes.POINTER(CWavelet), _d, ctypes.POINTER(CBins), _d,
                              _i, _vp, _vp, _vp, _vp, _i, _vp]),
    'ssqb_cwt_noalloc_max_bytes': (_sz, []),
    'ssqb_ridges_workspace_bytes': (_sz, [_i, _i, _i]),
    'ssqb_extract_ridges': (_i, [_vp, _i, _i, _vp, _vp, _d, _i, _i, _d, _i, _vp, _vp, _vp, _vp,
                                 _sz, _vp]),
    'ssqb_issq': (_i, [_vp, _i, _i, _vp, _vp, _i, _d, _i, _vp, _vp]),
    'ssqb_cwt_batch_workspace_bytes': (_sz, [_i, _i, _i]),
    'ssqb_cwt_batch': (_i, [_vp, _vp, _vp, _i, _i, _i, ctypes.POINTER(CWavelet), _d, _d,
                            _i, _vp, _vp, _vp, _sz, _vp]),
    'ssqb_cwt_batch_launches': (_i, [_vp, _i, _i, _i, _sz]),
    'ssqb_cwt_batch_ex': (_i, [_vp, _vp, _vp, _i, _i, _i, ctypes.POINTER(CWavelet), _d, _d,
                               _i, _vp, _vp, _vp, _sz, _i, _i, _vp]),
    'ssqb_cwt_batch_ex_launches': (_i, [_vp, _i, _i, _i, _sz, _i, _i]),
    'ssqb_cwt_band_rows': (_i, [_vp, _i, _i, ctypes.POINTER(CWavelet), _i, _i,
                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    'ssqb_cwt_adjoint_workspace_bytes': (_sz, [_i, _i, _i, _i]),
    'ssqb_cwt_adjoint': (_i, [_vp, _vp, _vp, _i, _vp, _i, _vp, _vp, _i, _i, _i, _i, _i,
                              _vp, _i, ctypes.POINTER(CWavelet), _i, _vp, _i, _vp, _sz,
                              _vp]),
    'ssqb_stft_adjoint_workspace_bytes': (_sz, [_i, _i, _i, _i, _i]),
    'ssqb_stft_adjoint': (_i, [_vp, _vp, _vp, _i, _vp, _i, _i, _i, _i, _i, _i, _i, _vp, _i,
                               _vp, _i, _vp, _sz, _vp]),
    'ssqb_phase_diff': (_i, [_vp, _i, _i, _i, _i, _i, _i, _i, _d, _d, _i, _vp, _vp]),
    'ssqb_trigdiff_workspace_bytes': (_sz, [_i, _i]),
    'ssqb_trigdiff': (_i, [_vp, _i, _i, _i, _i, _i, _d, _i, _i, _i, _vp, _vp, _sz, _vp]),
    'ssqb_istft_workspace_bytes': (_sz, [_i, _i, _i, _i]),
    'ssqb_istft': (_i, [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _d, _i, _vp, _vp, _sz, _vp]),
    'ssqb_squeeze_adjoint': (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _i, _i, _vp, _i, _vp]),
    'ssqb_icwt_adjoint': (_i, [_vp, _vp, _i, _i, _i, _i, _vp, _i, _vp]),
    'ssqb_squeeze_batch': (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp, _vp]),
}

# numpy layout of `ssqb_sig` (one signal of a batch of uneven lengths)
SIG_DTYPE = np.dtype([('x_off', np.int64), ('out_off', np.int64), ('idx_off', np.int64),
                      ('scales', np.uint64), ('weights', np.uint64),
                      ('N', np.int32), ('n1', np.int32), ('na', np.int32),
                      ('idx_pitch', np.int32), ('mode', np.int32), ('idx1', np.int32),
                      ('flipud', np.int32), ('nbins', np.int32), ('p', np.float64, (4,))],
                     align=True)
assert SIG_DTYPE.itemsize == 104

_lib = None
_lock = threading.Lock()


def load(path=LIB_PATH):
    """Load libssqb.so and declare its signatures (raises if missing)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise ImportError(
                    "ssqueezepy_b200: CUDA extension not built (%s missing); run "
                    "`python -m ssqueezepy_b200.build`" % path)
            lib = ctypes.CDLL(path)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(rc, what=''):
    if rc != OK:
        msg = load().ssqb_last_error().decode(errors='replace')
        exc = {EINVAL: ValueError, EUNSUPPORTED: NotImplementedError}.get(
            rc, RuntimeError)
        raise exc("ssqb%s failed (status %d): %s"
                  % (' ' + what if what else '', rc, msg))


def device_status(stream=None):
    """Read and clear the device status word (0 = ok)."""
    out = ctypes.c_int(0)
    check(load().ssqb_device_status(stream_ptr(stream), ctypes.byref(out)),
          'device_status')
    return out.value


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("ssqueezepy_b200 needs a CUDA device (B200, sm_100a); "
                           "there is no CPU fallback")
    load()


def stream_ptr(stream=None):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def make_wavelet(kind, p, band=(0., 0.), kc=None):
    w = CWavelet()
    w.kind = int(kind)
    for i, v in enumerate(p):
        w.p[i] = float(v)
    w.band[0], w.band[1] = float(band[0]), float(band[1])
    if kc is not None:
        w.npoly = len(kc)
        for m, v in enumerate(kc[:8]):
            w.kc[m] = float(v)
    return w


def wavelet_struct(wavelet):
    """The ssqb_wavelet of a `_params.Wavelet`: formula parameters, band and
    (higher-order GMW) Laguerre coefficients."""
    kind, *wp = wavelet.kernel_params()
    return make_wavelet(kind, wp, wavelet.band(), wavelet.poly())


def make_bins(mode, p, nbins, flipud):
    b = CBins()
    b.mode = int(mode)
    b.nbins = int(nbins)
    b.flipud = 1 if flipud else 0
    vals = list(p)
    b.idx1 = int(vals[4]) if len(vals) > 4 else 0
    for i in range(4):
        b.p[i] = float(vals[i])
    return b


def idx_pitch(n):
    """Row pitch of a bin-index buffer: n rounded up to 32 columns (64-byte
    aligned rows)."""
    return (n + 31) // 32 * 32


def exported_symbols():
    return list(SIGNATURES)
