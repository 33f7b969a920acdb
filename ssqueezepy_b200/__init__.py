# -*- coding: utf-8 -*-
"""B200-native synchrosqueezing hot path.

Drop-in replacements for ssqueezepy's `ssq_cwt`, `cwt`, `icwt`, `ssq_stft`,
`stft`, `istft` and `ssqueeze` (same signatures and return tuples), computed by the
hand-written sm_100a CUDA kernels of `_lib/libssqb.so` (C ABI:
include/ssqb.h). Host code only derives float64 parameters (scales,
frequencies, bin mapping); there is no CPU fallback.
"""
from ._transforms import (cwt, ssq_cwt, icwt, stft, istft, ssq_stft, ssqueeze, trigdiff,
                          phase_cwt, phase_cwt_num, phase_stft, issq_cwt, issq_stft, Wavelet,
                          configure)
from ._params import get_window_public as get_window
from ._params import (p2up, padsignal, process_scales, make_scales, cwt_scalebounds,
                      center_frequency, adm_ssq, logscale_transition_idx,
                      infer_scaletype, nv_from_scales)
from ._batch import SsqCwtBatch, ssq_cwt_batch
from ._ridges import extract_ridges
from . import _lib

__version__ = '0.1.0'
__all__ = ['cwt', 'ssq_cwt', 'icwt', 'stft', 'istft', 'ssq_stft', 'ssqueeze', 'get_window',
           'padsignal', 'trigdiff',
           'phase_cwt', 'phase_cwt_num', 'phase_stft', 'Wavelet', 'configure', 'p2up', 'process_scales',
           'make_scales', 'cwt_scalebounds', 'center_frequency', 'adm_ssq',
           'logscale_transition_idx', 'infer_scaletype', 'nv_from_scales',
           'SsqCwtBatch', 'ssq_cwt_batch', 'issq_cwt', 'issq_stft', 'extract_ridges']


def wavs():
    return Wavelet.SUPPORTED
