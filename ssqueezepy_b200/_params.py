# -*- coding: utf-8 -*-
"""Host-side float64 parameter math for the synchrosqueezing hot path.

Everything here runs once per call on the host, in float64, and produces the
small arrays and scalars the CUDA kernels consume: padding geometry, CWT
scales, synchrosqueezing frequencies (`ssq_freqs`), per-row squeeze weights
and the frequency-bin parameters.

The scale and frequency grids must come out bit-identical to ssqueezepy's so
that results can be compared with its float64 path element by element, so the
searches below walk the same sample grids as the reference routines they stand
in for (each function cites the one it follows). Unlike the reference, the
wavelet is always evaluated in float64 here, also for float32 transforms: the
reference's float32 `center_frequency` argmax can land on a neighbouring grid
point (ssqueezing.py:301-310, wavelets.py:714-717), which shifts `ssq_freqs`
and every bin decision with it.
"""
import numpy as np

pi = np.pi
EPS32 = float(np.finfo(np.float32).eps)
EPS64 = float(np.finfo(np.float64).eps)
LN2 = float(np.log(2))

# ssqueezepy/configs.ini defaults (wavelets.morlet, _gmw.gmw, _stft.stft,
# utils.cwt_utils.make_scales)
DEFAULTS = dict(morlet_mu=13.4, gmw_gamma=3., gmw_beta=60., gmw_norm='bandpass',
                wavelet_dtype='float32', stft_dtype='float32', downsample=4)


#### padding ##################################################################
def p2up(n):
    """Padded length and left/right pad (utils/common.py:32-51).

    Returns `(n_up, n1, n2)`: `n_up = 2**(1 + round(log2(n)))`,
    `n2 = (n_up - n)//2` on the right and `n1 = n_up - n - n2` on the left.
    """
    up = int(2 ** (1 + np.round(np.log2(n))))
    n2 = (up - n) // 2
    n1 = up - n - n2
    return up, int(n1), int(n2)


def pad_geometry(N, padlength=None):
    """`(n_up, n1, n2)` as chosen by utils/common.py:111-121."""
    if padlength is None:
        return p2up(N)
    n_up = int(padlength)
    if abs(n_up - N) % 2 == 0:
        n1 = n2 = (n_up - N) // 2
    else:
        n2 = (n_up - N) // 2
        n1 = n2 + 1
    return n_up, int(n1), int(n2)


PADTYPES = {'zero': 0, 'reflect': 1, 'symmetric': 2, 'replicate': 3, 'wrap': 4}


def process_fs_and_t(fs, t, N):
    """`(dt, fs, t)` as utils/cwt_utils.py:698-718."""
    if t is not None:
        t = np.asarray(t)
        if len(t) != N:
            raise Exception("`t` must be of same length as `x` "
                            "(%s != %s)" % (len(t), N))
        elif not np.mean(np.abs(np.diff(t, 2, axis=0))) < 1e-7:
            raise Exception("Time vector `t` must be uniformly sampled.")
        fs = 1 / (t[1] - t[0])
    else:
        if fs is None:
            fs = 1
        elif fs <= 0:
            raise ValueError("`fs` must be > 0")
    dt = 1 / fs
    return dt, fs, t


#### wavelets #################################################################
def xifn(scale, N):
    """Radian frequencies `[0, 1, ..., N//2, -(N - N//2 - 1), ..., -1]*2pi/N`
    times `scale` (wavelets.py:111-133, 473-484)."""
    h = (2 * pi) / N
    k = np.arange(N, dtype=np.float64)
    k[N // 2 + 1:] -= N
    xi = k * h
    return scale * xi


class Wavelet():
    """Frequency-domain wavelet: Morlet, or Generalized Morse (order 0, L1
    'bandpass' or L2 'energy' norm).

    Mirrors the parts of `ssqueezepy.Wavelet` (wavelets.py:14-470) the hot path
    uses: construction from a name or `(name, options)`, `dtype`, `config`,
    `fn(w)` and `__call__(scale=, N=)`. `fn` evaluates in float64 on the host
    and serves only the parameter searches; the transform evaluates the same
    formula on the GPU from `kernel_params()`.
    """
    SUPPORTED = {'gmw', 'morlet'}
    KIND_MORLET, KIND_GMW_L1, KIND_GMW_L2 = 0, 1, 2

    def __init__(self, wavelet='gmw', N=1024, dtype=None):
        name, opts = self._parse(wavelet)
        opts = dict(opts)
        if dtype is None:
            dtype = opts.pop('dtype', None)
        else:
            opts.pop('dtype', None)
        if name == 'morlet':
            mu = float(opts.pop('mu', DEFAULTS['morlet_mu']))
            if opts:
                raise TypeError("unsupported morlet options: %s" % list(opts))
            self.config = dict(mu=mu)
            self.kind = self.KIND_MORLET
        elif name == 'gmw':
            gamma = float(opts.pop('gamma', DEFAULTS['gmw_gamma']))
            beta = float(opts.pop('beta', DEFAULTS['gmw_beta']))
            norm = opts.pop('norm', DEFAULTS['gmw_norm'])
            order = opts.pop('order', 0)
            centered = opts.pop('centered_scale', False)
            if opts:
                raise TypeError("unsupported gmw options: %s" % list(opts))
            if gamma <= 0:
                raise ValueError(f"`gamma` must be positive (got {gamma})")
            if beta <= 0:
                raise ValueError(f"`beta` must be positive (got {beta})")
            if norm not in ('bandpass', 'energy'):
                raise ValueError("`norm` must be 'energy' or 'bandpass' "
                                 f"(got '{norm}')")
            if centered:
                raise NotImplementedError(
                    "GMW `centered_scale=True` is not on the accelerated path")
            order = _check_order(order)
            self.config = dict(gamma=gamma, beta=beta, norm=norm)
            if order != 0:
                self.config['order'] = order
            self.kind = (self.KIND_GMW_L1 if norm == 'bandpass' else
                         self.KIND_GMW_L2)
            if norm == 'energy':
                dtype = 'float64'  # wavelets.py:411-418
        else:
            raise ValueError("`wavelet` must be one of %s (got %s)"
                             % (sorted(self.SUPPORTED), name))
        self.name_ = name
        self._dtype = _dtype_str(dtype or DEFAULTS['wavelet_dtype'])
        self.N = N

    @staticmethod
    def _parse(wavelet):
        if isinstance(wavelet, Wavelet):
            return wavelet.name_, dict(wavelet.config, dtype=wavelet.dtype)
        if isinstance(wavelet, str):
            return wavelet.lower(), {}
        if isinstance(wavelet, tuple):
            if not (len(wavelet) == 2 and isinstance(wavelet[1], dict)):
                raise TypeError("`wavelet` tuple must be (name, dict)")
            return wavelet[0].lower(), wavelet[1]
        # a reference `ssqueezepy.Wavelet` instance: read its name and config
        cfg = getattr(wavelet, 'config', None)
        name = getattr(wavelet, 'name', None)
        if isinstance(cfg, dict) and isinstance(name, str):
            low = name.lower()
            if low.startswith('gmw'):
                cfg = {k: v for k, v in cfg.items()
                       if k in ('gamma', 'beta', 'norm', 'order',
                                'centered_scale')}
                cfg['dtype'] = getattr(wavelet, 'dtype', None)
                return 'gmw', cfg
            if low.startswith('morlet'):
                return 'morlet', dict(mu=cfg.get('mu', DEFAULTS['morlet_mu']),
                                      dtype=getattr(wavelet, 'dtype', None))
        raise TypeError("`wavelet` must be a name, (name, dict) or Wavelet "
                        "(got %s)" % type(wavelet))

    @classmethod
    def _init_if_not_isinstance(cls, wavelet, **kw):
        return wavelet if isinstance(wavelet, Wavelet) else cls(wavelet, **kw)

    @property
    def dtype(self):
        return self._dtype

    @property
    def order(self):
        return self.config.get('order', 0)

    def poly(self):
        """Laguerre coefficients kc of a higher-order GMW: psih = C(w) * base(w)
        with C(w) = sum_m kc[m] (2 w^gamma)^m and base the order-0 exponential
        without its norm constant (_gmw.py:268-296, 320-347). An order tuple
        averages the wavelets of its orders, i.e. their coefficient vectors
        (cwt_higher_order, _cwt.py:517-610, averages the transforms, which are
        linear in the wavelet). None for order 0."""
        order = self.order
        if order == 0 or self.kind == self.KIND_MORLET:
            return None
        c = self.config
        norm = c['norm']
        if isinstance(order, tuple):
            ks = [gmw_k_constants(c['gamma'], c['beta'], k, norm) for k in order]
            out = np.zeros(max(len(k) for k in ks))
            for k in ks:
                out[:len(k)] += k
            return out / len(ks)
        return gmw_k_constants(c['gamma'], c['beta'], order, norm)

    @property
    def name(self):
        if self.kind == self.KIND_MORLET:
            return 'Morlet'
        return 'GMW L1' if self.kind == self.KIND_GMW_L1 else 'GMW L2'

    @property
    def N(self):
        return self._N

    @N.setter
    def N(self, value):
        self._N = value
        self._xi = None

    @property
    def xi(self):
        if self._xi is None:
            self._xi = xifn(1., self._N)
        return self._xi

    # constants, float64 (wavelets.py:509-516, _gmw.py:191-195, 232-237)
    def constants(self):
        c = self.config
        if self.kind == self.KIND_MORLET:
            mu = c['mu']
            cs = (1 + np.exp(-mu**2) - 2 * np.exp(-3/4 * mu**2)) ** (-.5)
            ks = np.exp(-.5 * mu**2)
            return dict(mu=mu, ks=float(ks), C1=float(np.sqrt(2) * cs * pi**.25))
        gamma, beta = c['gamma'], c['beta']
        wc = (beta / gamma) ** (1 / gamma)  # _gmw.py:638
        if self.kind == self.KIND_GMW_L1:
            return dict(gamma=gamma, beta=beta, wc=float(wc),
                        wcl=float(np.log(wc)))
        from scipy.special import gamma as gamma_fn
        r = (2 * beta + 1) / gamma
        norm = float(np.sqrt(2. * pi * gamma * 2.**r / gamma_fn(r)))
        return dict(gamma=gamma, beta=beta, wc=float(wc), l2norm=norm)

    def fn(self, w):
        """psih(w), float64 (wavelets.py:521-527, _gmw.py:203-210, 246-251)."""
        w = np.atleast_1d(np.asarray(w, dtype=np.float64))
        k = self.constants()
        if self.kind == self.KIND_MORLET:
            return k['C1'] * (np.exp(-.5 * (w - k['mu'])**2)
                              - k['ks'] * np.exp(-.5 * w**2))
        nonneg = (w >= 0)
        w = w * nonneg
        kc = self.poly()
        if kc is not None:
            y = 2 * w**k['gamma']
            C = np.zeros_like(w)
            for m in range(len(kc)):
                C = C + kc[m] * y**m
            with np.errstate(divide='ignore'):
                if self.kind == self.KIND_GMW_L1:
                    e = (-k['beta'] * k['wcl'] + k['wc']**k['gamma']
                         + k['beta'] * np.log(w) - w**k['gamma'])
                else:
                    e = k['beta'] * np.log(w) - w**k['gamma']
                return C * np.exp(e) * nonneg
        with np.errstate(divide='ignore'):
            if self.kind == self.KIND_GMW_L1:
                return 2 * np.exp(-k['beta'] * k['wcl'] + k['wc']**k['gamma']
                                  + k['beta'] * np.log(w) - w**k['gamma']
                                  ) * nonneg
            return (k['l2norm'] * w**k['beta'] * np.exp(-w**k['gamma'])
                    * nonneg)

    def __call__(self, w=None, *, scale=None, N=None, nohalf=True):
        if w is not None:
            psih = self.fn(w)
        else:
            if scale is None:
                scale = 1.
            scale = np.asarray(scale, dtype=np.float64)
            if scale.ndim >= 1 and scale.size > 1:
                scale = scale.reshape(-1, 1)
            xi = xifn(1., N) if N is not None else self.xi
            psih = self.fn(scale * xi)
        if not nohalf:
            n = psih.shape[-1]
            if n % 2 == 0:
                psih[..., n // 2] /= 2
        return psih

    def band(self, log_floor=-69.):
        """(w_lo, w_hi): outside this interval |psih(w)| < e^log_floor times
        its peak (e^-69 ~ 1e-30), so the kernels skip evaluating it there."""
        k = self.constants()
        if self.kind == self.KIND_MORLET:
            mu = k['mu']
            r = np.sqrt(-2 * log_floor)
            neg = np.sqrt(max(0., -2 * log_floor - mu**2))
            return (min(mu - r, -neg), mu + r)
        g, b, wc = k['gamma'], k['beta'], k['wc']
        # memoized: the transforms build their wavelets per call
        key = (self.kind, tuple(sorted(self.config.items())), float(log_floor))
        hit = _BANDS.get(key)
        if hit is not None:
            return hit
        if len(_BANDS) > 256:
            _BANDS.clear()
        if self.poly() is not None:
            # a polynomial factor moves the peak: scan log|psih| on a fine
            # log grid and widen by a grid step on each side
            w = np.geomspace(1e-8 * wc, 1e3 * wc, 1 << 16)
            with np.errstate(divide='ignore'):
                lp = np.log(np.abs(self.fn(w)))
            keep = np.nonzero(lp >= lp.max() + log_floor)[0]
            i0, i1 = max(keep[0] - 1, 0), min(keep[-1] + 1, len(w) - 1)
            _BANDS[key] = (float(w[i0]), float(w[i1]))
            return _BANDS[key]

        def e(w):  # log of psih relative to its peak at wc
            return b * np.log(w / wc) - (w**g - wc**g)
        lo, hi = 1e-300, wc
        for _ in range(200):
            mid = np.sqrt(lo * hi)
            lo, hi = (mid, hi) if e(mid) < log_floor else (lo, mid)
        w_lo = lo
        lo, hi = wc, wc * 2
        while e(hi) > log_floor:
            hi *= 2
        for _ in range(200):
            mid = .5 * (lo + hi)
            lo, hi = (mid, hi) if e(mid) > log_floor else (lo, mid)
        _BANDS[key] = (w_lo, hi)
        return _BANDS[key]

    def kernel_params(self):
        """(kind, p0, p1, p2, p3) passed to the CUDA kernels."""
        k = self.constants()
        if self.kind == self.KIND_MORLET:
            return (self.kind, k['mu'], k['ks'], k['C1'], 0.)
        if self.kind == self.KIND_GMW_L1:
            return (self.kind, k['gamma'], k['beta'], k['wc'], k['wcl'])
        return (self.kind, k['gamma'], k['beta'], k['wc'], k['l2norm'])


MAX_GMW_ORDER = 7
_BANDS = {}   # (kind, config, log_floor) -> band of a GMW


def _check_order(order):
    if isinstance(order, (list, range)):
        order = tuple(order)
    if isinstance(order, tuple):
        order = tuple(int(k) for k in order)
        if len(order) == 1:
            order = order[0]
    ks = order if isinstance(order, tuple) else (int(order),)
    if any(k < 0 or k > MAX_GMW_ORDER for k in ks):
        raise NotImplementedError("GMW orders 0..%d are on the accelerated path "
                                  "(got %s)" % (MAX_GMW_ORDER, order))
    return order if isinstance(order, tuple) else int(order)


def gmw_k_constants(gamma, beta, k, norm='bandpass'):
    """Laguerre polynomial constants times the order-k norm, float64
    (_gmw.py:368-396): L_m = (-1)^m Gamma(k+c+1) / (Gamma(c+m+1) Gamma(k-m+1))
    / m!, c = r - 1, r = (2 beta + 1) / gamma; times sqrt(Gamma(r) k! /
    Gamma(k+r)) and 2 (bandpass), or sqrt(2 pi gamma 2^r k! / Gamma(k+r))
    (energy)."""
    from scipy.special import gammaln, gamma as gamma_fn
    r = (2 * beta + 1) / gamma
    c = r - 1
    if norm == 'bandpass':
        coeff = np.sqrt(np.exp(gammaln(r) + gammaln(k + 1) - gammaln(k + r)))
    else:
        coeff = np.sqrt(2 * pi * gamma * (2**r) * np.exp(gammaln(k + 1) - gammaln(k + r)))
    L = np.zeros(k + 1)
    for m in range(k + 1):
        fact = np.exp(gammaln(k + c + 1) - gammaln(c + m + 1) - gammaln(k - m + 1))
        L[m] = (-1)**m * fact / gamma_fn(m + 1)
    kc = L * coeff
    if norm == 'bandpass':
        kc = kc * 2
    return kc


def _dtype_str(dtype):
    s = str(np.dtype(dtype)) if not isinstance(dtype, str) else dtype
    s = s.split('.')[-1]
    if s not in ('float32', 'float64'):
        raise ValueError("`dtype` must be float32 or float64 (got %s)" % s)
    return s


def process_gmw_wavelet(wavelet, l1_norm):
    """GMW norm follows `l1_norm` (_cwt.py:497-514)."""
    norm = 'bandpass' if l1_norm else 'energy'
    if isinstance(wavelet, str) and wavelet.lower()[:3] == 'gmw':
        return ('gmw', {'norm': norm})
    if isinstance(wavelet, tuple) and wavelet[0].lower()[:3] == 'gmw':
        name, opts = wavelet
        opts = dict(opts)
        opts['norm'] = opts.get('norm', norm)
        return (name, opts)
    if isinstance(wavelet, Wavelet):
        if wavelet.name == 'GMW L2' and l1_norm:
            raise ValueError("using GMW L2 wavelet with `l1_norm=True`")
        elif wavelet.name == 'GMW L1' and not l1_norm:
            raise ValueError("using GMW L1 wavelet with `l1_norm=False`")
    return wavelet


#### grid searches (algos.py:616-703) #########################################
def _first_below(arr, th):
    """Index of first element `< th`, else the last index (algos.py:616-622)."""
    hit = np.nonzero(arr < th)[0]
    return int(hit[0]) if hit.size else len(arr) - 1


def find_maximum(fn, step_size=1e-3, steps_per_search=1e4, step_start=0,
                 step_limit=1000, min_value=-1):
    """Scan `|fn|` on consecutive `linspace` windows of `steps_per_search`
    points until a window's max stops growing (algos.py:625-662)."""
    n = int(steps_per_search)
    incr = int(n * step_size)
    best, best_at = min_value, None
    s = 0
    while True:
        lo = step_start + incr * s
        grid = np.linspace(lo, lo + incr, n, endpoint=False)
        vals = np.abs(fn(grid))
        m = vals.max()
        if m > best:
            best, best_at = m, grid[np.argmax(vals)]
        elif m < best:
            break
        s += 1
        if grid.max() > step_limit:
            raise ValueError("could not find function maximum below %s"
                             % step_limit)
    return best_at, best


def find_first_occurrence(fn, value, step_size=1e-3, steps_per_search=1e4,
                          step_start=0, step_limit=1000):
    """Earliest grid point where `|fn|` reaches `value` within one grid step
    of the window's largest jump (algos.py:665-703)."""
    n = int(steps_per_search)
    incr = int(n * step_size)
    s = 0
    while True:
        lo = step_start + incr * s
        grid = np.linspace(lo, lo + incr, n, endpoint=False)
        over = grid.max() > step_limit
        if over:
            grid = np.clip(grid, None, step_limit)
        vals = np.abs(fn(grid))
        jump = np.abs(np.diff(vals)).max()
        dist = np.abs(vals - value)
        if np.any(dist <= jump):
            i = int(np.argmin(dist))
            return grid[i], vals[i]
        s += 1
        if over:
            raise ValueError("could not find input value to yield %s" % value)


#### center frequency (wavelets.py:611-750, 951-964) ##########################
def _aifftshift(v):
    n = len(v)
    if n % 2:
        return np.fft.ifftshift(v)
    h = n // 2
    return np.concatenate([v[h + 1:], v[:h + 1]])


def center_frequency(wavelet, scale=None, N=1024, kind='energy',
                     force_int=None):
    """Radian center frequency at `scale` ('peak', 'energy' with force_int,
    'peak-ct')."""
    if kind not in ('energy', 'peak', 'peak-ct'):
        raise ValueError("`kind` must be one of energy, peak, peak-ct")
    wavelet = Wavelet._init_if_not_isinstance(wavelet)
    if kind == 'peak-ct':
        return float(find_maximum(wavelet.fn)[0])
    if scale is None:
        scale = (4 / pi) * find_maximum(wavelet.fn)[0]
    w = _aifftshift(xifn(1., N))
    psih = wavelet.fn(np.asarray(scale) * w)
    apsih2 = np.abs(psih)**2
    if kind == 'peak':
        return float(w[np.argmax(apsih2)])
    if force_int is False:
        wc_ct = find_maximum(wavelet.fn)[0]
        sc = (4 / pi) * wc_ct
        psih = wavelet.fn(np.asarray(sc) * w)
        apsih2 = np.abs(psih)**2
        wc = _trapz(apsih2 * w) / _trapz(apsih2)
        return float(wc * (sc / scale))
    return float(_trapz(apsih2 * w) / _trapz(apsih2))


def _trapz(y, x=None):
    """Composite trapezoid rule (unit spacing if `x` is None). Each panel is
    halved before the sum, as scipy.integrate.trapezoid does: halving a
    subnormal panel is inexact, so the order matters for bit parity."""
    y = np.asarray(y)
    d = 1 if x is None else np.diff(x)
    return (d * (y[1:] + y[:-1]) / 2.0).sum()


#### scale bounds & scales (utils/cwt_utils.py) ###############################
def find_min_scale(wavelet, cutoff=1):
    """cwt_utils.py:412-431."""
    w_peak, peak = find_maximum(wavelet.fn)
    if cutoff > 0:
        start, limit = w_peak, 10 * w_peak
    else:
        start, limit = 0, w_peak
    w_cut, _ = find_first_occurrence(wavelet.fn, value=abs(cutoff) * peak,
                                     step_start=start, step_limit=limit)
    return w_cut / pi


def find_max_scale(wavelet, N, bin_loc=1, bin_amp=1):
    """cwt_utils.py:434-456."""
    wc_ct = center_frequency(wavelet, kind='peak-ct', N=N)
    scalec_ct = (4 / pi) * wc_ct
    psih = wavelet(scale=scalec_ct, N=N)[:N // 2 + 1]
    xi = xifn(scalec_ct, N)
    midx = np.argmax(psih)
    w_bin = xi[np.nonzero(psih[:midx] < psih.max() * bin_amp)[0][-1]]
    return scalec_ct * (w_bin / xi[bin_loc])


def find_max_scale_alt(wavelet, N, min_cutoff=.1, max_cutoff=.8):
    """cwt_utils.py:630-695: smallest bin spacing whose grid lands
    symmetrically about the wavelet's peak."""
    if max_cutoff <= 0 or min_cutoff <= 0:
        raise ValueError("`max_cutoff` and `min_cutoff` must be positive")
    elif max_cutoff <= min_cutoff:
        raise ValueError("must have `max_cutoff > min_cutoff`")
    w_peak, peak = find_maximum(wavelet.fn)
    w_cut, _ = find_first_occurrence(wavelet.fn, value=min_cutoff * peak,
                                     step_start=0, step_limit=w_peak)
    w_ltp = np.arange(w_cut, w_peak, step=1 / N)
    div_size = (w_peak - w_ltp[:-1]) * 2
    n_divs = w_ltp[:-1] / div_size
    hits = np.nonzero(np.diff(n_divs % 1) < -.8)[0]
    if hits.size == 0:
        raise Exception("Failed to find suffciently-integer xi divisions; try "
                        "widening (min_cutoff, max_cutoff)")
    div_scale = div_size[hits[0] + 1]
    w_1div = pi / (N / 2)
    return div_scale / w_1div


def cwt_scalebounds(wavelet, N, preset=None, use_padded_N=True):
    """`(min_scale, max_scale)` for presets 'maximal' / 'minimal' / None /
    'naive' (cwt_utils.py:66-188, default cutoffs :127, :155-157)."""
    if preset not in (None, 'maximal', 'minimal', 'naive'):
        raise ValueError("`preset` must be one of maximal, minimal, naive")
    if preset == 'naive':
        return 1, N
    M = p2up(N)[0] if use_padded_N else N
    min_scale = find_min_scale(wavelet, cutoff=-.5)
    if preset == 'maximal':
        max_scale = find_max_scale(wavelet, M, bin_loc=2, bin_amp=1)
    else:
        max_scale = find_max_scale_alt(wavelet, M, min_cutoff=.6, max_cutoff=.8)
    return min_scale, max_scale


def find_downsampling_scale(wavelet, scales, span=5, tol=3, nonzero_th=.02,
                            nonzero_tol=4., N=2048):
    """First scale group whose wavelet peaks crowd within `tol` bins of their
    joint peak ('sum' criterion; cwt_utils.py:459-580)."""
    Psih = wavelet(scale=scales, N=N)
    Psih = Psih[:, :Psih.shape[1] // 2]
    n_groups = len(Psih) - span - 1
    i = 0
    for i in range(n_groups):
        g = Psih[i:i + span]
        gmax = g.max(axis=1)[:, None]
        if (g > nonzero_th * gmax).sum() / span > nonzero_tol:
            continue
        cols = np.nonzero(g == gmax)[1]
        joint = np.argmax(np.prod(g, 0))
        if np.abs(cols - joint).sum() < tol:
            break
    return i if (i < n_groups - 1) else None


def make_scales(N, min_scale=None, max_scale=None, nv=32, scaletype='log',
                wavelet=None, downsample=None):
    """cwt_utils.py:301-372."""
    if scaletype == 'log-piecewise' and wavelet is None:
        raise ValueError("must pass `wavelet` for `scaletype == 'log-piecewise'`")
    if min_scale is None and max_scale is None and wavelet is not None:
        min_scale, max_scale = cwt_scalebounds(wavelet, N, use_padded_N=True)
    else:
        min_scale = min_scale or 1
        max_scale = max_scale or N
    downsample = int(downsample if downsample is not None else
                     DEFAULTS['downsample'])
    na = int(np.ceil(nv * np.log2(max_scale / min_scale)))
    mn_pow = int(np.floor(nv * np.log2(min_scale)))
    mx_pow = mn_pow + na
    if scaletype == 'log':
        scales = 2 ** (np.arange(mn_pow, mx_pow) / nv)
    elif scaletype == 'log-piecewise':
        scales = 2 ** (np.arange(mn_pow, mx_pow) / nv)
        idx = find_downsampling_scale(wavelet, scales)
        if idx is not None:
            scales = np.hstack([scales[:idx],
                                scales[idx + downsample - 1::downsample]])
    elif scaletype == 'linear':
        min_scale, max_scale = 2**(mn_pow / nv), 2**(mx_pow / nv)
        na = int(np.ceil(max_scale / min_scale))
        scales = np.linspace(min_scale, max_scale, na)
    else:
        raise ValueError("`scaletype` must be 'log' or 'linear'; "
                         "got: %s" % scaletype)
    return scales.reshape(-1, 1)


def logscale_transition_idx(scales):
    """Index splitting two log-spaced pieces, or None (cwt_utils.py:375-394)."""
    scales = np.asarray(scales)
    d2 = np.abs(np.diff(np.log(scales), 2, axis=0))
    idx = int(np.argmax(d2)) + 2
    d2max = d2.max()
    d2[idx - 2] = 0
    th = 1e-14 if scales.dtype == np.float64 else 1e-6
    if not np.any(d2max > 100 * np.abs(d2).mean()):
        return None
    elif not np.all(np.abs(d2) < th):
        return None
    return idx


def nv_from_scales(scales):
    """Per-row voices, shape (na, 1) (cwt_utils.py:397-409)."""
    scales = np.asarray(scales)
    logdiffs = 1 / np.diff(np.log2(scales), axis=0)
    return np.vstack([logdiffs[:1], logdiffs])


def infer_scaletype(scales):
    """'log' / 'linear' / 'log-piecewise' and nv (cwt_utils.py:264-298)."""
    scales = np.asarray(scales).reshape(-1, 1)
    if scales.dtype not in (np.float32, np.float64):
        raise TypeError("`scales.dtype` must be np.float32 or np.float64 "
                        "(got %s)" % scales.dtype)
    th_log = 4e-15 if scales.dtype == np.float64 else 8e-7
    th_lin = th_log * 1e3
    if np.mean(np.abs(np.diff(np.log(scales), 2, axis=0))) < th_log:
        nv = int(np.round(1 / np.diff(np.log2(scales), axis=0)[0].squeeze()))
        return 'log', nv
    elif np.mean(np.abs(np.diff(scales, 2, axis=0))) < th_lin:
        return 'linear', None
    elif logscale_transition_idx(scales) is None:
        raise ValueError("could not infer `scaletype` from `scales`; "
                         "`scales` array must be linear or exponential.")
    return 'log-piecewise', nv_from_scales(scales)


def process_scales(scales, N, wavelet=None, nv=None, get_params=False,
                   use_padded_N=True):
    """Scales (na, 1) float64 from a scheme string or an array
    (cwt_utils.py:196-261)."""
    preset = None
    if isinstance(scales, str):
        if ':' in scales:
            scales, preset = scales.split(':')
        elif scales == 'log-piecewise':
            preset = 'maximal'
        if scales not in ('log', 'log-piecewise', 'linear'):
            raise ValueError("`scales` must be one of log, log-piecewise, "
                             "linear (got %s)" % scales)
        if nv is None:
            nv = 32
        if wavelet is None:
            raise ValueError("must set `wavelet` if `scales` isn't array")
        scaletype = scales
    else:
        arr = _to_numpy(scales)
        if arr.squeeze().ndim != 1:
            raise ValueError("`scales`, if array, must be 1D "
                             "(got shape %s)" % str(arr.shape))
        scaletype, _nv = infer_scaletype(arr)
        if scaletype == 'log':
            if nv is not None and _nv != nv:
                raise Exception("`nv` used in `scales` differs from "
                                "`nv` passed (%s != %s)" % (_nv, nv))
            nv = _nv
        elif scaletype == 'log-piecewise':
            nv = _nv
        arr = arr.reshape(-1, 1)
        if nv is not None and not isinstance(nv, np.ndarray):
            nv = int(nv)
        return arr if not get_params else (arr, scaletype, len(arr), nv)

    if nv is not None:
        if not (nv > 0 and float(nv).is_integer()):
            raise ValueError(f"'nv' must be a positive integer (got {nv})")
        nv = int(nv)
    wavelet = Wavelet._init_if_not_isinstance(wavelet)
    mn, mx = cwt_scalebounds(wavelet, N=N, preset=preset,
                             use_padded_N=use_padded_N)
    out = make_scales(N, mn, mx, nv=nv, scaletype=scaletype, wavelet=wavelet)
    return out if not get_params else (out, scaletype, len(out), nv)


def _to_numpy(a):
    if hasattr(a, 'detach'):
        a = a.detach().cpu().numpy()
    return np.asarray(a)


#### synchrosqueezing frequencies (ssqueezing.py:228-310) ####################
def _get_center_frequency(wavelet, N, maprange, dt, scale, was_padded):
    if was_padded:
        N = p2up(N)[0]
    wc = center_frequency(wavelet, N=N, scale=scale, kind=maprange,
                          force_int=True if maprange == 'energy' else None)
    return wc / (2 * pi) / dt


def ssq_freqrange(maprange, dt, N, wavelet, scales, was_padded):
    if isinstance(maprange, (tuple, list)):
        return maprange[0], maprange[1]
    if maprange == 'maximal':
        return 1 / (dt * N), 1 / (2 * dt)
    kw = dict(wavelet=wavelet, N=N, maprange=maprange, dt=dt,
              was_padded=was_padded)
    return (_get_center_frequency(**kw, scale=scales[-1]),
            _get_center_frequency(**kw, scale=scales[0]))


def _exp_fm(t, fmin, fmax):
    tmin, tmax = t.min(), t.max()
    a = (fmin**tmax / fmax**tmin) ** (1 / (tmax - tmin))
    b = fmax**(1 / tmax) * (1 / a)**(1 / tmax)
    return a * b**t


def compute_associated_frequencies(scales, N, wavelet, ssq_scaletype, maprange,
                                   was_padded=True, dt=1, transform='cwt'):
    """Ascending `ssq_freqs` (ssqueezing.py:247-291)."""
    fm, fM = ssq_freqrange(maprange, dt, N, wavelet, scales, was_padded)
    na = len(scales)
    if ssq_scaletype == 'log':
        return fm * np.power(fM / fm, np.arange(na) / (na - 1))
    if ssq_scaletype == 'log-piecewise':
        idx = logscale_transition_idx(scales)
        if idx is None:
            return fm * np.power(fM / fm, np.arange(na) / (na - 1))
        f1 = _get_center_frequency(wavelet, N, maprange, dt, scales[idx],
                                   was_padded)
        t1 = np.arange(0, na - idx - 1) / (na - 1)
        t2 = np.arange(na - idx - 1, na) / (na - 1)
        t1 = np.hstack([t1, t2[0]])
        sqf = np.hstack([_exp_fm(t1, fm, f1)[:-1], _exp_fm(t2, f1, fM)])
        sidx = logscale_transition_idx(sqf)
        if sidx is None:
            raise Exception("couldn't find logscale transition index of "
                            "generated `ssq_freqs`; something went wrong")
        assert (na - sidx) == idx, "{} != {}".format(na - sidx, idx)
        return sqf
    if transform == 'cwt':
        return np.linspace(fm, fM, na)
    return np.linspace(0, .5, na) / dt


def _nonzero_nonneg(x):
    return EPS64 if x < EPS64 else x


def bin_params(ssq_freqs, logscale):
    """Bin mapping of the squeeze (algos.py:81-87, 356-374).

    Returns `(mode, p)`: mode 0 = log (p = vlmin, dvl), 1 = log-piecewise
    (p = vlmin0, vlmin1, dvl0, dvl1, idx1), 2 = linear (p = vmin, dv).
    """
    v = np.asarray(ssq_freqs, dtype=np.float64).ravel()
    if not logscale:
        dv = _nonzero_nonneg(float(v[1] - v[0]))
        return 2, (float(v[0]), dv, 0., 0., 0)
    idx = logscale_transition_idx(v)
    vlmin = float(np.log2(v[0]))
    if idx is None:
        dvl = _nonzero_nonneg(float(np.log2(v[1]) - np.log2(v[0])))
        return 0, (vlmin, dvl, 0., 0., 0)
    vlmin1 = float(np.log2(v[idx - 1]))
    dvl0 = _nonzero_nonneg(float(np.log2(v[1]) - np.log2(v[0])))
    dvl1 = _nonzero_nonneg(float(np.log2(v[idx]) - np.log2(v[idx - 1])))
    return 1, (vlmin, vlmin1, dvl0, dvl1, int(idx - 1))


def squeeze_weights(scales, cwt_scaletype, nv, transform, ssq_freqs=None):
    """Per-row weight `const_i` of `Tx[k, j] += Wx[i, j]*const_i`
    (ssqueezing.py:124-134)."""
    na = len(scales) if scales is not None else len(ssq_freqs)
    if transform == 'stft':
        v = np.asarray(ssq_freqs)
        return np.full(na, float(v[1] - v[0]))
    if cwt_scaletype.startswith('log'):
        c = LN2 / np.asarray(nv, dtype=np.float64)
        return np.broadcast_to(c, (na, 1)).reshape(-1).astype(np.float64)
    s = np.asarray(scales, dtype=np.float64).ravel()
    return (s[1] - s[0]) / s


#### icwt (_cwt.py:441-450, utils/cwt_utils.py:28-47, 583-627) ###############
def integrate_analytic(int_fn):
    """Trapezoid integral over (0, inf) of a function decaying to the right,
    with the near-zero part on a log grid (cwt_utils.py:583-627)."""
    t0 = np.logspace(-15, -1, 1000)
    int_nz = _trapz(int_fn(t0), t0)
    for m, mxlim in zip([1, 1, 4, 8], [1, 20, 80, 160]):
        n = 10000 * m
        t = np.linspace(mxlim, .1, n, endpoint=False)[::-1].copy()
        arr = int_fn(t)
        mi = int(np.argmax(arr))
        cut = _first_below(np.abs(arr[mi:]), 1e-15) + mi
        if (len(t) - cut > 1000 * m) and np.sum(np.abs(arr)) > 1e-5:
            break
    else:
        if int_nz < 1e-5:
            raise Exception("Could not find converging or non-negligibly"
                            "-valued bounds of integration for `int_fn`")
    return _trapz(arr[:cut], t[:cut]) + int_nz


def adm_ssq(wavelet):
    """Synchrosqueezing admissibility constant, integral psih(w)/w."""
    wavelet = Wavelet._init_if_not_isinstance(wavelet)
    with np.errstate(divide='ignore', invalid='ignore'):
        c = integrate_analytic(lambda w: np.conj(wavelet.fn(w)) / w)
    return float(np.real(c))


#### STFT window (_stft.py:259-310) ###########################################
def get_window(window, win_len, n_fft=None, derivative=False):
    """Window padded to `n_fft` and its frequency-domain derivative, float64."""
    from scipy import signal as sig
    if n_fft is None:
        pl, pr = 0, 0
    else:
        if win_len > n_fft:
            raise ValueError("Can't have `win_len > n_fft` ({} > {})".format(
                win_len, n_fft))
        pl = (n_fft - win_len) // 2
        pr = (n_fft - win_len - pl)
    if window is not None:
        if isinstance(window, str):
            window = sig.get_window(window, win_len, fftbins=True)
        elif isinstance(window, np.ndarray) or hasattr(window, 'detach'):
            window = _to_numpy(window).astype(np.float64)
        else:
            raise ValueError("`window` must be string or np.ndarray "
                             "(got %s)" % window)
    else:
        window = sig.windows.dpss(win_len, max(4, win_len // 8), sym=False)
    window = np.asarray(window, dtype=np.float64)
    if len(window) < (win_len + pl + pr):
        window = np.pad(window, [pl, pr])
    diff_window = None
    if derivative:
        from scipy import fft as sfft
        Nw = len(window)
        xi = xifn(1., Nw)
        if Nw % 2 == 0:
            xi[Nw // 2] = 0
        diff_window = sfft.ifft(sfft.fft(window) * 1j * xi).real
    return window, diff_window


def get_window_public(window, win_len, n_fft=None, derivative=False, dtype=None):
    """`get_window` of _stft.py:259-310: the window padded to `n_fft` (and its
    frequency-domain derivative), cast to `dtype` (default: float64, the
    window's own) with denormals zeroed."""
    if isinstance(window, np.ndarray) and len(window) != win_len:
        import warnings
        warnings.warn("len(window) != win_len (%s != %s)" % (len(window), win_len))
    win, dwin = get_window(window, win_len, n_fft, derivative=derivative)
    dt = _dtype_str(dtype) if dtype is not None else 'float64'
    win = zero_denormals(win.astype(dt))
    if derivative:
        return win, zero_denormals(dwin.astype(dt))
    return win


def padsignal(x, padtype='reflect', padlength=None, get_params=False):
    """`padsignal` of utils/common.py:54-158: pad the last axis of a 1D / 2D
    numpy array or torch tensor to `padlength` (default: `p2up`), left pad n1,
    right pad n2. numpy arrays take all five modes on the host (np.pad, and
    the edge-repeating 'symmetric' by reversal); tensors take 'zero' and
    'reflect' on their device, as the reference allows."""
    is_numpy = isinstance(x, np.ndarray)
    supported = (('zero', 'reflect', 'symmetric', 'replicate', 'wrap') if is_numpy
                 else ('zero', 'reflect'))
    if padtype not in supported:
        raise ValueError("`padtype` must be one of: %s (got %s)"
                         % (', '.join(supported), padtype))
    if not hasattr(x, 'ndim'):
        raise TypeError("`x` must be a numpy array or torch Tensor (got %s)" % type(x))
    if x.ndim not in (1, 2):
        raise ValueError("`x` must be 1D or 2D (got x.ndim == %s)" % x.ndim)
    n_up, n1, n2 = pad_geometry(x.shape[-1], padlength)
    if is_numpy:
        pw = (n1, n2) if x.ndim == 1 else [(0, 0), (n1, n2)]
        if padtype == 'symmetric':
            r = x[..., ::-1]
            xp = np.concatenate([r[..., r.shape[-1] - n1:] if n1 else r[..., :0], x,
                                 r[..., :n2]], axis=-1)
        else:
            mode = {'zero': 'constant', 'reflect': 'reflect', 'replicate': 'edge',
                    'wrap': 'wrap'}[padtype]
            xp = np.pad(x, pw, mode=mode)
    else:
        import torch
        mode = 'constant' if padtype == 'zero' else 'reflect'
        xp = (torch.nn.functional.pad(x[None], (n1, n2), mode)[0] if x.ndim == 1 else
              torch.nn.functional.pad(x, (n1, n2), mode))
    return (xp, n_up, n1, n2) if get_params else xp


def zero_denormals(x):
    """Zero |x| < 1000*tiny (algos.py:593-612)."""
    tiny = 1000 * np.finfo(x.dtype).tiny
    x[(x < tiny) & (x > -tiny)] = 0
    return x
