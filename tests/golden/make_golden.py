# -*- coding: utf-8 -*-
"""Generate the golden fixtures under tests/golden/ by running ssqueezepy
itself (float64 path, CPU, numba) on seeded inputs.

Usage (needs the ssqueezepy source tree; only run where it exists):

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py \
        /path/to/ssqueezepy-checkout

Writes:
  host_params.npz  scales / ssq_freqs / bin parameters / adm_ssq for many
                   (wavelet, N, scheme) combinations
  transforms.npz   small end-to-end ssq_cwt / cwt / ssq_stft / stft / icwt
                   outputs (float64) with their inputs
  digests.npz      full-size (N=10,000 and N=160,000) float64 digests: row
                   norms and row sums of Wx and Tx, total norms, and a bin
                   histogram, for size-independent checks
  issq.npz         issq_cwt / issq_stft of seeded complex Tx (rebuilt from
                   the seed by the tests), full and per-component inversion

  ridges.npz       extract_ridges (serial code path) of a seeded synthetic
                   Tf with two ridges, float64 and float32, log and linear
                   frequency axes, with its inputs

  higher.npz       higher-order GMW transforms (float64, N=256): cwt with
                   order=2, cwt averaged over orders (0, 1, 2), ssq_cwt with
                   order=(0, 1), and order-1 / order-3 wavelet samples

  istft.npz        istft of stft outputs and of seeded complex one-sided
                   spectra: hop, win_len < n_fft, win_exp 0 / 1 / 2,
                   modulated on and off, float64 and float32, with inputs

  difftype.npz     ssq_cwt with difftype 'phase' and 'numeric' (difforder
                   1, 2, 4), get_w=True, float64, and phase_cwt /
                   phase_cwt_num of the same Wx

  squeezing.npz    ssq_cwt / ssq_stft with squeezing 'lebesgue', 'abs' and a
                   function (W * W), with and without get_w, float64

  utils.npz        padsignal (five modes, default and given lengths) and
                   get_window (with derivative) outputs; trigdiff of seeded
                   complex rows (default reflect padding without N, zero
                   padding with N, already padded 2D and 3D input)

  stft_any.npz     stft (Sx, dSx) and ssq_stft (Tx) for n_fft that are not
                   powers of two (598, 121, 120, 100), modulated on and off,
                   hop 1 to 4, float64

`--only issq` / `--only ridges` / `--only higher` / `--only istft` /
`--only difftype` / `--only squeezing` / `--only utils` / `--only stft_any`
writes that file alone.
"""
import os
import sys
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def chirp_signal(N, seed=0):
    """Linear chirp 0.01->0.2 cycles/sample + AM tone at 0.3 + N(0, 0.1^2)
    noise; the 10k / 160k single-signal workload."""
    t = np.arange(N, dtype=np.float64)
    rng = np.random.default_rng(seed)
    x = (np.cos(2 * np.pi * (0.01 * t + 0.19 * t**2 / (2 * N)))
         + (0.5 + 0.5 * np.cos(2 * np.pi * 0.001 * t)) * np.cos(2 * np.pi * 0.3 * t)
         + 0.1 * rng.standard_normal(N))
    return x


def main(ref_root):
    os.environ['SSQ_GPU'] = '0'
    os.environ.setdefault('SSQ_PARALLEL', '1')
    sys.path.insert(0, ref_root)
    import ssqueezepy as sq
    from ssqueezepy import Wavelet
    from ssqueezepy.utils import (process_scales, p2up, adm_ssq,
                                  logscale_transition_idx)
    from ssqueezepy.ssqueezing import _compute_associated_frequencies
    from ssqueezepy.algos import _get_params_find_closest_log

    wavs = {
        'morlet6': ('morlet', {'mu': 6.}),
        'morlet13.4': ('morlet', {'mu': 13.4}),
        'morlet5': ('morlet', {'mu': 5.}),
        'gmw3_60': ('gmw', {'gamma': 3., 'beta': 60.}),
        'gmw3_8': ('gmw', {'gamma': 3., 'beta': 8.}),
    }

    def W(key):
        name, opts = wavs[key]
        return Wavelet((name, dict(opts, dtype='float64')))

    #### host params ##########################################################
    hp = {}
    Ns = [64, 100, 256, 300, 1000, 2048, 4096, 10000, 16384, 65536, 160000,
          1048576]
    for key in wavs:
        w = W(key)
        hp[f'adm_ssq/{key}'] = np.array(adm_ssq(w))
        for N in Ns:
            hp[f'p2up/{N}'] = np.array(p2up(N))
            for st in ('log', 'log-piecewise', 'linear', 'log:maximal',
                       'log:minimal'):
                try:
                    s = process_scales(st, N, w, nv=32)
                except Exception:
                    hp[f'scales/{key}/{N}/{st}'] = np.array([])  # raises
                    continue
                s1 = s.ravel()
                if s1.size > 2048:  # long linear grids: keep ends + digest
                    hp[f'scales_digest/{key}/{N}/{st}'] = np.array(
                        [s1.size, s1.sum(), (s1 * s1).sum()])
                    s1 = np.hstack([s1[:64], s1[-64:]])
                hp[f'scales/{key}/{N}/{st}'] = s1
                if N not in (256, 10000, 160000):
                    continue
                for sqs in ('log', 'log-piecewise', 'linear'):
                    for mr in ('peak', 'energy', 'maximal'):
                        if mr == 'maximal' and sqs == 'log-piecewise':
                            continue
                        try:
                            f = _compute_associated_frequencies(
                                s, N, w, sqs, mr, True, 1., 'cwt')
                        except Exception:
                            continue
                        k = f'ssq_freqs/{key}/{N}/{st}/{sqs}/{mr}'
                        hp[k] = (f if f.size <= 2048 else
                                 np.hstack([f[:64], f[-64:]]))
                        if sqs.startswith('log'):
                            _, p = _get_params_find_closest_log(f)
                            hp['binp/' + k[10:]] = np.array(
                                [float(v) for v in p.values()])
        hp[f'nv32/{key}'] = np.array(32)
    np.savez_compressed(os.path.join(HERE, 'host_params.npz'), **hp)
    print('host_params', len(hp))

    #### small end-to-end transforms ########################################
    tr = {}
    cases = [
        # name, N, wavelet, scales, ssq_freqs, maprange, padtype, flipud
        ('c0', 256, 'morlet6', 'log-piecewise', 'log', 'peak', 'reflect', True),
        ('c1', 160, 'gmw3_60', 'log-piecewise', None, 'peak', 'reflect', True),
        ('c2', 150, 'morlet13.4', 'log', 'log', 'maximal', 'zero', True),
        ('c3', 100, 'gmw3_60', 'linear', 'linear', 'energy', 'reflect', False),
        ('c4', 200, 'morlet6', 'log:maximal', 'log', 'peak', 'reflect', True),
    ]
    for name, N, wk, st, sqf, mr, pad, flip in cases:
        x = chirp_signal(N, seed=len(name) * 7 + N)
        w = W(wk)
        Tx, Wx, ssq_freqs, scales, wph, dWx = sq.ssq_cwt(
            x, w, scales=st, nv=32, ssq_freqs=sqf, maprange=mr, padtype=pad,
            flipud=flip, get_w=True, get_dWx=True)
        Tx2, *_ = sq.ssq_cwt(x, w, scales=st, nv=32, ssq_freqs=sqf,
                             maprange=mr, padtype=pad, flipud=flip)
        assert np.allclose(Tx, Tx2, atol=1e-12)
        tr[f'{name}/x'] = x
        tr[f'{name}/meta'] = np.array([N, 32], dtype=np.int64)
        tr[f'{name}/cfg'] = np.array([wk, st, str(sqf), mr, pad, str(flip)])
        tr[f'{name}/Tx'] = Tx2
        tr[f'{name}/Wx'] = Wx
        if name == 'c0':
            tr[f'{name}/w'] = wph
        tr[f'{name}/ssq_freqs'] = np.asarray(ssq_freqs)
        tr[f'{name}/scales'] = np.asarray(scales).ravel()
        tr[f'{name}/icwt'] = sq.icwt(Wx, w, scales=scales, x_mean=x.mean())
    # batched (equal length), matches looped per the reference tests
    xb = np.stack([chirp_signal(100, seed=s) for s in (11, 12)])
    w = W('morlet6')
    Tx, Wx, f, s = sq.ssq_cwt(xb, w, scales='log-piecewise', nv=32,
                              ssq_freqs='log')
    tr['b0/x'], tr['b0/Tx'], tr['b0/Wx'] = xb, Tx, Wx
    tr['b0/ssq_freqs'], tr['b0/scales'] = np.asarray(f), np.asarray(s).ravel()

    # STFT
    stft_cases = [('s0', 512, 'hann', 128, 128, 1),
                  ('s1', 300, 'hann', 64, 48, 1),
                  ('s2', 256, None, 64, 64, 1),
                  ('s3', 400, 'hann', 64, 64, 3)]
    for name, N, win, n_fft, win_len, hop in stft_cases:
        x = chirp_signal(N, seed=N + 3)
        Tx, Sx, ssq_freqs, Sfs, wph, dSx = sq.ssq_stft(
            x, window=win, n_fft=n_fft, win_len=win_len, hop_len=hop,
            dtype='float64', get_w=True, get_dWx=True)
        Tx2, *_ = sq.ssq_stft(x, window=win, n_fft=n_fft, win_len=win_len,
                              hop_len=hop, dtype='float64')
        tr[f'{name}/x'] = x
        tr[f'{name}/cfg'] = np.array([str(win), n_fft, win_len, hop])
        tr[f'{name}/Tx'], tr[f'{name}/Sx'] = Tx2, Sx
        if name == 's0':
            tr[f'{name}/w'] = wph
        tr[f'{name}/Sfs'] = np.asarray(Sfs)
    np.savez_compressed(os.path.join(HERE, 'transforms.npz'), **tr)
    print('transforms', len(tr))

    #### full-size digests ####################################################
    dg = {}
    for name, N, wk, sqf in (('d10k', 10000, 'morlet6', 'log'),
                             ('d160k', 160000, 'gmw3_60', None)):
        x = chirp_signal(N, seed=0)
        w = W(wk)
        Tx, Wx, ssq_freqs, scales, wph = sq.ssq_cwt(
            x, w, scales='log-piecewise', nv=32, ssq_freqs=sqf, get_w=True)
        dg[f'{name}/Wx_rownorm'] = np.linalg.norm(Wx, axis=1)
        dg[f'{name}/Wx_rowsum'] = Wx.sum(axis=1)
        dg[f'{name}/Tx_rownorm'] = np.linalg.norm(Tx, axis=1)
        dg[f'{name}/Tx_rowsum'] = Tx.sum(axis=1)
        dg[f'{name}/Tx_colsum_stride'] = Tx.sum(axis=0)[::97]
        dg[f'{name}/Wx_row'] = Wx[len(Wx) // 3][::16]
        dg[f'{name}/Tx_row'] = Tx[np.argmax(np.linalg.norm(Tx, axis=1))][::16]
        dg[f'{name}/Tx_row_idx'] = np.array(np.argmax(np.linalg.norm(Tx, axis=1)))
        dg[f'{name}/ssq_freqs'] = np.asarray(ssq_freqs)
        dg[f'{name}/scales'] = np.asarray(scales).ravel()
        fin = np.isfinite(wph)
        dg[f'{name}/w_finite'] = np.array(fin.sum())
        dg[f'{name}/w_sum'] = np.array(wph[fin].sum())
        print(name, Tx.shape)
    np.savez_compressed(os.path.join(HERE, 'digests.npz'), **dg)


def issq_inputs():
    """Seeded complex Tx (CWT-like 120 x 700, STFT-like 129 x 700) and curve
    centres / widths (700, 2) with some columns marked -1 (no curve)."""
    rng = np.random.default_rng(77)
    Tc = rng.standard_normal((120, 700)) + 1j * rng.standard_normal((120, 700))
    Ts = rng.standard_normal((129, 700)) + 1j * rng.standard_normal((129, 700))
    cc = rng.integers(0, 120, (700, 2))
    cc[rng.random((700, 2)) < 0.1] = -1
    cw = rng.integers(0, 12, (700, 2))
    return Tc, Ts, cc, cw


def issq_fixtures(ref_root):
    os.environ['SSQ_GPU'] = '0'
    sys.path.insert(0, ref_root)
    import ssqueezepy as sq
    Tc, Ts, cc, cw = issq_inputs()
    out = {}
    for key, (name, opts) in (('gmw', ('gmw', {})), ('morlet6', ('morlet', {'mu': 6.}))):
        w = sq.Wavelet((name, dict(opts, dtype='float64')))  # float64 admissibility
        out['cwt_full_' + key] = sq.issq_cwt(Tc, w)
        out['cwt_comp_' + key] = sq.issq_cwt(Tc, w, cc, cw)
    out['stft_full_hann256'] = sq.issq_stft(Ts, 'hann', n_fft=256)
    out['stft_comp_hann256'] = sq.issq_stft(Ts, 'hann', cc=cc, cw=cw, n_fft=256)
    np.savez_compressed(os.path.join(HERE, 'issq.npz'), **out)


def ridges_fixtures(ref_root):
    """Tf (64 x 400): two ridges (a rising and a falling frequency track,
    amplitudes 1 and 0.6) over complex noise of 0.05; scales geomspace(1, 50)
    for the log axis, linspace(0, 0.5) for the linear one."""
    sys.path.insert(0, ref_root)
    from ssqueezepy.ridge_extraction import extract_ridges
    rng = np.random.default_rng(31)
    nf, N = 64, 400
    t = np.arange(N)
    f = np.arange(nf)[:, None]
    c1 = 10 + 40 * t / N
    c2 = 55 - 30 * (t / N) ** 2
    Tf = (np.exp(-(f - c1) ** 2 / 6) + 0.6 * np.exp(-(f - c2) ** 2 / 4)
          + 0.05 * (rng.standard_normal((nf, N)) + 1j * rng.standard_normal((nf, N))))
    Tf = Tf * np.exp(1j * rng.uniform(0, 2 * np.pi, (nf, N)))
    out = dict(Tf=Tf, scales_log=np.geomspace(1, 50, nf), scales_lin=np.linspace(0, .5, nf))
    for dt in ('f64', 'f32'):
        T = Tf if dt == 'f64' else Tf.astype(np.complex64)
        for ax, tr in (('log', 'cwt'), ('lin', 'stft')):
            sc = out['scales_' + ax]
            for nr, bw in ((1, 15), (2, 4)):
                key = '%s_%s_r%d' % (dt, ax, nr)
                i, fr, e = extract_ridges(T, sc, penalty=2., n_ridges=nr, bw=bw, transform=tr,
                                          get_params=True, parallel=False)
                out[key + '_idx'], out[key + '_f'], out[key + '_e'] = i, fr, e
    np.savez_compressed(os.path.join(HERE, 'ridges.npz'), **out)


def higher_fixtures(ref_root):
    os.environ['SSQ_GPU'] = '0'
    sys.path.insert(0, ref_root)
    import ssqueezepy as sq
    from ssqueezepy import Wavelet
    x = chirp_signal(256, seed=4)
    out = dict(x=x)
    w = Wavelet(('gmw', dict(dtype='float64')))
    Wx, sc = sq.cwt(x, w, order=2, astensor=False)
    out['cwt_o2_Wx'], out['scales'] = Wx, sc
    Wx, _ = sq.cwt(x, w, order=(0, 1, 2), astensor=False)
    out['cwt_avg012_Wx'] = Wx
    Tx, Wx, f, _ = sq.ssq_cwt(x, w, order=(0, 1), astensor=False)
    out['ssq_avg01_Tx'], out['ssq_avg01_f'] = Tx, f
    w1 = Wavelet(('gmw', dict(order=1, dtype='float64')))
    out['psih_w'] = np.linspace(0, 12, 257)
    out['psih_o1'] = np.asarray(w1(out['psih_w'])).ravel()
    w3e = Wavelet(('gmw', dict(order=3, norm='energy', dtype='float64')))
    out['psih_o3e'] = np.asarray(w3e(out['psih_w'])).ravel()
    np.savez_compressed(os.path.join(HERE, 'higher.npz'), **out)


ISTFT_CASES = [
    # name, N (signal; None: the spectrum is seeded noise), n_fft, win_len,
    # hop, window, N passed to istft, modulated, win_exp, dtype
    ('a', 300, 64, 64, 1, 'hann', 300, True, 1, 'float64'),
    ('b', 301, 64, 48, 4, 'hann', 301, True, 0, 'float64'),
    ('c', None, 64, 64, 3, 'hann', None, False, 1, 'float64'),
    ('d', None, 32, 32, 2, None, None, True, 2, 'float64'),
    ('e', 300, 64, 64, 1, 'hann', 300, True, 1, 'float32'),
    ('f', 600, 512, 512, 4, 'hann', 600, True, 1, 'float64'),
    ('g', 1000, 128, 100, 5, 'hamming', 997, False, 1, 'float64'),
    # n_fft not a power of two (the reference's benchmark length, odd, even)
    ('h', 600, 598, 598, 4, 'hann', 600, True, 1, 'float64'),
    ('i', 300, 121, 121, 3, 'hann', 300, True, 1, 'float64'),
    ('j', 300, 100, 90, 2, 'hann', 300, False, 0, 'float64'),
    ('k', 300, 121, 121, 1, 'hann', 300, True, 1, 'float32'),
]


def istft_fixtures(ref_root):
    os.environ['SSQ_GPU'] = '0'
    sys.path.insert(0, ref_root)
    import ssqueezepy as sq
    out = {}
    for name, N, n_fft, win_len, hop, win, Ni, mod, wexp, dt in ISTFT_CASES:
        if N is not None:
            x = chirp_signal(N, seed=len(name) + N)
            Sx = sq.stft(x, window=win, n_fft=n_fft, win_len=win_len, hop_len=hop,
                         modulated=mod, dtype='float64')
            Sx = np.asarray(Sx)
        else:
            rng = np.random.default_rng(n_fft + hop)
            shape = (n_fft // 2 + 1, 80)
            Sx = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        if dt == 'float32':
            Sx = Sx.astype(np.complex64)
        xr = sq.istft(Sx, window=win, n_fft=n_fft, win_len=win_len, hop_len=hop,
                      N=Ni, modulated=mod, win_exp=wexp)
        out[name + '/Sx'] = Sx
        out[name + '/x'] = np.asarray(xr)
    np.savez_compressed(os.path.join(HERE, 'istft.npz'), **out)


def difftype_fixtures(ref_root):
    os.environ['SSQ_GPU'] = '0'
    sys.path.insert(0, ref_root)
    import ssqueezepy as sq
    from ssqueezepy import Wavelet
    from ssqueezepy._ssq_cwt import phase_cwt, phase_cwt_num
    x = chirp_signal(256, seed=6)
    out = dict(x=x)
    w = Wavelet(('gmw', dict(dtype='float64')))
    Tx, Wx, f, sc, wp = sq.ssq_cwt(x, w, nv=8, difftype='phase', get_w=True,
                                   astensor=False)
    out.update({'phase/Tx': Tx, 'phase/f': f, 'phase/w': wp})
    for k in (1, 2, 4):
        Tx, Wx, f, sc, wn = sq.ssq_cwt(x, w, nv=8, difftype='numeric', difforder=k,
                                       get_w=True, astensor=False)
        out.update({'num%d/Tx' % k: Tx, 'num%d/w' % k: wn, 'num%d/f' % k: f})
    # the returned Wx of difftype='numeric' is the padded transform less 4
    # columns on each side (_ssq_cwt.py:294-296)
    out['num4/Wx_shape'] = np.array(Wx.shape)
    out['num4/Wx_row0'] = Wx[0]
    W0, _ = sq.cwt(x, w, nv=8, astensor=False)
    out['cwt/Wx'] = W0
    out['phase_cwt/w'] = phase_cwt(W0, None, difftype='phase')
    out['phase_cwt_num/w'] = phase_cwt_num(W0, 1., difforder=4)
    np.savez_compressed(os.path.join(HERE, 'difftype.npz'), **out)


def square(W):
    """A squeezing function that works on numpy arrays and torch tensors."""
    return W * W


def squeezing_fixtures(ref_root):
    os.environ['SSQ_GPU'] = '0'
    sys.path.insert(0, ref_root)
    import ssqueezepy as sq
    from ssqueezepy import Wavelet
    x = chirp_signal(256, seed=8)
    out = dict(x=x)
    w = Wavelet(('gmw', dict(dtype='float64')))
    for name, sqz in (('lebesgue', 'lebesgue'), ('abs', 'abs'), ('square', square)):
        Tx, *_ = sq.ssq_cwt(x, w, nv=8, squeezing=sqz, astensor=False)
        out['cwt_%s/Tx' % name] = Tx
        Tx, *_ = sq.ssq_cwt(x, w, nv=8, squeezing=sqz, get_w=True, astensor=False)
        out['cwt_%s_w/Tx' % name] = Tx
        Tx, *_ = sq.ssq_stft(x, 'hann', n_fft=64, squeezing=sqz, dtype='float64',
                             astensor=False)
        out['stft_%s/Tx' % name] = Tx
    np.savez_compressed(os.path.join(HERE, 'squeezing.npz'), **out)


PAD_CASES = [(pt, pl) for pt in ('zero', 'reflect', 'symmetric', 'replicate', 'wrap')
             for pl in (None, 64, 77)]
WINDOW_CASES = [('hann', 64, None), ('hamming', 48, 64), (None, 64, None)]


def utils_fixtures(ref_root):
    os.environ['SSQ_GPU'] = '0'
    sys.path.insert(0, ref_root)
    import ssqueezepy as sq
    from ssqueezepy.utils import padsignal
    x = np.random.default_rng(21).standard_normal((3, 37))
    out = dict(x=x)
    for pt, pl in PAD_CASES:
        xp, n_up, n1, n2 = padsignal(x, pt, pl, get_params=True)
        out['pad_%s_%s' % (pt, pl)] = xp
        out['pad_%s_%s_geom' % (pt, pl)] = np.array([n_up, n1, n2])
    for win, wl, nf in WINDOW_CASES:
        w, dw = sq.get_window(win, wl, nf, derivative=True)
        out['win_%s_%d_%s' % (win, wl, nf)] = w
        out['dwin_%s_%d_%s' % (win, wl, nf)] = dw
    from ssqueezepy.utils import trigdiff
    rng = np.random.default_rng(22)
    A = rng.standard_normal((5, 300)) + 1j * rng.standard_normal((5, 300))
    Ap = rng.standard_normal((2, 3, 512)) + 1j * rng.standard_normal((2, 3, 512))
    out['td_A'], out['td_Ap'] = A, Ap
    out['td_reflect'] = trigdiff(A, fs=2.)
    out['td_zero_N'] = trigdiff(A, fs=1., padtype='zero', N=300)
    out['td_rpadded'] = trigdiff(Ap[0], fs=3., rpadded=True, N=300)
    out['td_rpadded3'] = trigdiff(Ap, rpadded=True, N=256, n1=100)
    np.savez_compressed(os.path.join(HERE, 'utils.npz'), **out)


STFT_ANY_CASES = [  # name, N, n_fft, hop, modulated, window
    ('n598', 600, 598, 4, True, 'hann'),
    ('n121', 300, 121, 3, True, 'hann'),
    ('n120', 300, 120, 1, False, 'hann'),
    ('n100', 300, 100, 2, True, None),
]


def stft_any_fixtures(ref_root):
    os.environ['SSQ_GPU'] = '0'
    sys.path.insert(0, ref_root)
    import ssqueezepy as sq
    out = {}
    for name, N, n_fft, hop, mod, win in STFT_ANY_CASES:
        x = chirp_signal(N, seed=n_fft)
        Sx, dSx = sq.stft(x, window=win, n_fft=n_fft, hop_len=hop, modulated=mod,
                          derivative=True, dtype='float64')
        Tx, *_ = sq.ssq_stft(x, window=win, n_fft=n_fft, hop_len=hop, modulated=mod,
                             dtype='float64', astensor=False)
        out[name + '/x'], out[name + '/Sx'] = x, np.asarray(Sx)
        out[name + '/dSx'], out[name + '/Tx'] = np.asarray(dSx), np.asarray(Tx)
    np.savez_compressed(os.path.join(HERE, 'stft_any.npz'), **out)


if __name__ == '__main__':
    args = [a for a in sys.argv[1:] if not a.startswith('--')]
    root = args[0] if args else '/root/reference'
    if '--only' in sys.argv and 'issq' in sys.argv:
        issq_fixtures(root)
    elif '--only' in sys.argv and 'ridges' in sys.argv:
        ridges_fixtures(root)
    elif '--only' in sys.argv and 'higher' in sys.argv:
        higher_fixtures(root)
    elif '--only' in sys.argv and 'istft' in sys.argv:
        istft_fixtures(root)
    elif '--only' in sys.argv and 'difftype' in sys.argv:
        difftype_fixtures(root)
    elif '--only' in sys.argv and 'squeezing' in sys.argv:
        squeezing_fixtures(root)
    elif '--only' in sys.argv and 'utils' in sys.argv:
        utils_fixtures(root)
    elif '--only' in sys.argv and 'stft_any' in sys.argv:
        stft_any_fixtures(root)
    else:
        main(root)
        issq_fixtures(root)
        ridges_fixtures(root)
        higher_fixtures(root)
        istft_fixtures(root)
        difftype_fixtures(root)
        squeezing_fixtures(root)
        utils_fixtures(root)
        stft_any_fixtures(root)
