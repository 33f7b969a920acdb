// Prologue/epilogue operators for the tile FFT kernels: padded-signal FFT
// (x_hat), fused CWT (wavelet x x_hat -> Wx, dWx -> phase transform -> bin),
// fused STFT (framing + windows -> Sx, dSx -> phase transform -> bin).
#pragma once
#include "tile_kernels.cuh"

namespace ssqb {

// ---- parameters passed by value ------------------------------------------
struct WavDev {
  int kind;          // 0 Morlet, 1 GMW L1 (bandpass), 2 GMW L2 (energy)
  double p0, p1, p2, p3;  // Morlet: mu, ks, C1; GMW: gamma, beta, wc, wcl | l2norm
  double wcg;        // GMW: wc^gamma
  double lo, hi;     // psih = 0 outside [lo, hi] (skipped when lo >= hi)
  int ibeta;         // GMW L1: beta when it is an integer in [0, 128], else -1
  int npoly;         // GMW order > 0: the factor 2 | l2norm becomes C(2 w^gamma)
  double kc[8];      // C's coefficients, zero from npoly on
};

// Higher-order GMW factor C = sum_m kc[m] y^m, y = 2 x^gamma (Horner; the
// zero coefficients past npoly leave it exact)
__device__ __forceinline__ double gmw_poly(const WavDev& w, double xg) {
  const double y = 2.0 * xg;
  double c = w.kc[7];
#pragma unroll
  for (int m = 6; m >= 0; --m) c = fma(c, y, w.kc[m]);
  return c;
}

// x^n for 0 <= n < 256 by binary powering (relative error ~ a few ulps)
__device__ __forceinline__ double powi(double x, int n) {
  double r = 1.0, p = x;
#pragma unroll
  for (int bit = 0; bit < 8; ++bit) {
    if (n & (1 << bit)) r *= p;
    p *= p;
  }
  return r;
}

struct BinDev {
  int mode;          // 0 log, 1 log-piecewise, 2 linear
  int idx1;
  int flipud;
  int nbins;         // omax + 1
  double p0, p1, p2, p3;  // log: vlmin, dvl | piecewise: vlmin0, vlmin1, dvl0, dvl1 | lin: vmin, dv
};

// Per-signal descriptor of a batch of uneven lengths (same layout as
// ssqb_sig in include/ssqb.h).
struct SigDesc {
  long long x_off, out_off, idx_off;
  const double* scales;
  const double* weights;
  int N, n1, na, idx_pitch;
  int mode, idx1, flipud, nbins;
  double p0, p1, p2, p3;
};

constexpr uint16_t kNoBin = 0xFFFF;
constexpr double kTwoPi = 6.283185307179586;  // the literal of algos.py:867

// ---- padding index map (utils/common.py:54-158) -------------------------
// q: position relative to x[0]; returns the source index, or -1 for a zero.
enum PadType { PAD_ZERO = 0, PAD_REFLECT = 1, PAD_SYMMETRIC = 2, PAD_REPLICATE = 3,
               PAD_WRAP = 4, PAD_NONE = 5 };

__device__ __forceinline__ int pad_src(long long q, int N, int padtype) {
  if (q >= 0 && q < N) return (int)q;
  switch (padtype) {
    case PAD_REFLECT: {  // numpy 'reflect': period 2(N-1), no edge repeat
      if (N == 1) return 0;
      long long P = 2LL * (N - 1);
      long long r = q % P;
      if (r < 0) r += P;
      return (int)(r >= N ? P - r : r);
    }
    case PAD_SYMMETRIC: {  // edge repeated: period 2N
      long long P = 2LL * N;
      long long r = q % P;
      if (r < 0) r += P;
      return (int)(r >= N ? P - 1 - r : r);
    }
    case PAD_REPLICATE:
      return q < 0 ? 0 : N - 1;
    case PAD_WRAP: {
      long long r = q % N;
      if (r < 0) r += N;
      return (int)r;
    }
    default:
      return -1;
  }
}

// ---- wavelets, float64 (wavelets.py:521-527, _gmw.py:203-210, 246-251) --
// Formula branches; psih_fp64 picks one per call.
__device__ __forceinline__ double psih_morlet(const WavDev& w, double x) {
  // C1 (ea - ks ec), ea = exp(-(x-mu)^2/2), ec = exp(-x^2/2). The ratio of
  // the two terms is ks ec / ea = exp(-mu x): where mu |x| >= 40 the
  // smaller one is below 2^-57 of the larger, under a quarter ulp, and
  // the difference rounds to the larger term alone, so its exp is skipped.
  const double mx = w.p0 * x;
  const double d = x - w.p0;
  const double a = -0.5 * (d * d);
  const double c = -0.5 * (x * x);
  const double ea = (a > -708.0 && mx > -40.0) ? exp(a) : 0.0;
  const double ec = (c > -708.0 && mx < 40.0) ? exp(c) : 0.0;
  return w.p2 * (ea - w.p1 * ec);
}

// GMW L1 with gamma = 3 and an integer beta: 2 exp(beta ln(x/wc) - (x^3 -
// wc^3)) = 2 (x/wc)^beta exp(wc^3 - x^3), x > 0
__device__ __forceinline__ double psih_gmw3(const WavDev& w, double x) {
  const double x3 = x * x * x;
  const double e = w.wcg - x3;
  if (!(e > -708.0)) return 0.0;
  const double f = w.npoly ? gmw_poly(w, x3) : 2.0;
  return f * powi(x / w.p2, w.ibeta) * exp(e);
}

// GMW L1 / L2, any gamma and beta, x > 0
__device__ __forceinline__ double psih_gmw(const WavDev& w, double x) {
  const double lw = log(x);
  const double xg = (w.p0 == 3.0) ? x * x * x : exp(w.p0 * lw);
  if (w.kind == 1) {
    const double e = -w.p1 * w.p3 + w.wcg + w.p1 * lw - xg;
    if (!(e > -708.0)) return 0.0;
    return (w.npoly ? gmw_poly(w, xg) : 2.0) * exp(e);
  }
  // L2: norm * x^beta * exp(-x^gamma)
  const double e = w.p1 * lw - xg;
  if (!(e > -708.0)) return 0.0;
  return (w.npoly ? gmw_poly(w, xg) : w.p3) * exp(e);
}

// 0 Morlet, 1 GMW L1 gamma 3 integer beta, 2 other GMW
__device__ __forceinline__ int psih_kind_of(const WavDev& w) {
  if (w.kind == 0) return 0;
  return (w.kind == 1 && w.ibeta >= 0 && w.p0 == 3.0) ? 1 : 2;
}

template <int KIND>
__device__ __forceinline__ double psih_kind(const WavDev& w, double x) {
  if (w.lo < w.hi && (x < w.lo || x > w.hi)) return 0.0;
  if constexpr (KIND == 0) {
    return psih_morlet(w, x);
  } else {
    if (x <= 0.0) return 0.0;
    if constexpr (KIND == 1) return psih_gmw3(w, x);
    else return psih_gmw(w, x);
  }
}

__device__ __forceinline__ double psih_fp64(const WavDev& w, double x) {
  const int k = psih_kind_of(w);
  if (k == 0) return psih_kind<0>(w, x);
  if (k == 1) return psih_kind<1>(w, x);
  return psih_kind<2>(w, x);
}

// ---- frequency bin (algos.py:859-953; round = half-to-even, as numba) ----
__device__ __forceinline__ int bin_of(const BinDev& bp, double w) {
  const double omax = (double)(bp.nbins - 1);
  double k;
  if (bp.mode == 2) {
    k = fmin(rint(fmax((w - bp.p0) / bp.p1, 0.0)), omax);
  } else {
    const double wl = log2(w);
    if (bp.mode == 0) {
      k = fmin(rint(fmax((wl - bp.p0) / bp.p1, 0.0)), omax);
    } else if (wl > bp.p1) {
      k = fmin(rint((wl - bp.p1) / bp.p3) + (double)bp.idx1, omax);
    } else {
      k = fmax(rint((wl - bp.p0) / bp.p2), 0.0);
    }
  }
  int ki = (int)k;
  if (bp.flipud) ki = bp.nbins - 1 - ki;
  return ki;
}

// Bin position in float32 with a guard band: returns the bin, or -2 when
// the position lies within kBinGuard of a rounding edge (or of the
// log-piecewise split), where only the float64 decision is trusted. The
// float32 position carries ~1e-5 bins of error at most here (phase transform
// ~1e-7 relative -> ~5e-6 bins; log2f and the float32 affine map ~2e-5).
constexpr float kBinGuard = 2.5e-4f;
__device__ __forceinline__ int bin_of_fast(const BinDev& bp, float w) {
  const float omax = (float)(bp.nbins - 1);
  float pos, lo_clamp = 0.f;
  int add = 0;
  if (bp.mode == 2) {
    pos = (w - (float)bp.p0) * (float)(1.0 / bp.p1);
  } else {
    const float wl = log2f(w);
    if (bp.mode == 0) {
      pos = (wl - (float)bp.p0) * (float)(1.0 / bp.p1);
    } else {
      const float split = (float)bp.p1;  // vlmin1
      if (fabsf(wl - split) < 1e-4f * fmaxf(1.f, fabsf(split))) return -2;
      if (wl > split) {
        pos = (wl - split) * (float)(1.0 / bp.p3);
        add = bp.idx1;
        lo_clamp = -3.0e38f;
      } else {
        pos = (wl - (float)bp.p0) * (float)(1.0 / bp.p2);
      }
    }
  }
  const float fr = pos - floorf(pos);
  if (!(fabsf(fr - 0.5f) >= kBinGuard)) return -2;  // also catches NaN
  const float k = fminf(fmaxf(rintf(pos), lo_clamp) + (float)add, omax);
  int ki = (int)fmaxf(k, 0.f);
  if (bp.mode == 1 && add == 0) ki = (int)fmaxf(rintf(pos), 0.f);
  if (bp.flipud) ki = bp.nbins - 1 - ki;
  return ki;
}

// Phase transform and bin of one (Wx, dWx) pair (algos.py:864-876): w =
// |Im(dWx conj Wx)| / (|Wx|^2 2pi), Sfs shift for the STFT (algos.py:963-964).
// The bin is decided in float32 when that is safe, else in float64; either
// way it equals the float64 decision from these values. Returns kNoBin where
// |Wx| <= gamma.
// The phase transform alone (inf where |Wx| < gamma), for outputs that ask
// for w without a bin index.
template <typename C>
__device__ __forceinline__ double phase_w(C Wv, C dWv, double sfs, bool stft, double gamma) {
  const double c = Wv.x, d = Wv.y, a = dWv.x, b = dWv.y;
  const double m2 = c * c + d * d;
  const double ph = (b * c - a * d) / (m2 * kTwoPi);
  const double wv = stft ? fabs(sfs - ph) : fabs(ph);
  return (m2 < gamma * gamma) ? __longlong_as_double(0x7ff0000000000000ULL) : wv;
}

template <typename C>
__device__ __forceinline__ uint16_t phase_bin(C Wv, C dWv, double sfs, bool stft,
                                              const BinDev& bp, double gamma,
                                              int* status, double* w_out) {
  const double c = Wv.x, d = Wv.y, a = dWv.x, b = dWv.y;
  const double m2 = c * c + d * d;
  const double num = b * c - a * d;
  const bool keep = m2 > gamma * gamma;  // |Wx| > gamma
  if (w_out) *w_out = phase_w(Wv, dWv, sfs, stft, gamma);
  if (!keep) return kNoBin;
  int k = -2;
  {
    const float ph32 = (float)num / ((float)m2 * 6.2831855f);
    const float w32 = stft ? fabsf((float)sfs - ph32) : fabsf(ph32);
    if (w32 > 0.f && w32 < 3.0e38f) k = bin_of_fast(bp, w32);
  }
  if (k == -2) {
    const double ph = num / (m2 * kTwoPi);
    const double w = stft ? fabs(sfs - ph) : fabs(ph);
    k = bin_of(bp, w);
  }
  if (k < 0 || k >= bp.nbins || k >= (int)kNoBin) {
    set_status(status, DEV_BAD_BIN);
    return kNoBin;
  }
  return (uint16_t)k;
}

template <typename C> __device__ __forceinline__ void put_w(C* p, double v);
template <> __device__ __forceinline__ void put_w<float2>(float2* p, double v) {
  reinterpret_cast<float*>(p)[0] = (float)v;
}
template <> __device__ __forceinline__ void put_w<double2>(double2* p, double v) {
  reinterpret_cast<double*>(p)[0] = v;
}

// ---- x_hat: FFT of the padded signal, float64 ------------------------------
template <typename TX>
struct XhatOp {
  static constexpr int NARR = 1;
  static constexpr bool kDirect = true;
  static constexpr bool kBatch = false;
  const TX* x;       // (B, N)
  double2* xh;       // (B, Npad)
  int N, Npad, n1, padtype;
  __device__ XhatOp bind(int) const { return *this; }
  __device__ int rows() const { return 1; }
  __device__ void load(int b, int, int k, double2 (&v)[1]) const {
    const int s = pad_src((long long)k - n1, N, padtype);
    v[0] = make_double2(s >= 0 ? (double)x[(size_t)b * N + s] : 0.0, 0.0);
  }
  __device__ void store(int b, int, int n, double2 (&v)[1]) const {
    xh[(size_t)b * Npad + n] = v[0];
  }
};

// ---- fused CWT ---------------------------------------------------------------
// C: arithmetic type of the transform; OC: stored type of Wx / dWx / w.
template <typename OC> __device__ __forceinline__ OC out_c(double2 v);
template <> __device__ __forceinline__ float2 out_c<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
template <> __device__ __forceinline__ double2 out_c<double2>(double2 v) { return v; }
template <typename OC> __device__ __forceinline__ OC out_c(float2 v);
template <> __device__ __forceinline__ float2 out_c<float2>(float2 v) { return v; }

// ---- trigdiff (utils/common.py:161-245): D = ifft(fft(pad(A)) * i xi fs) ------
// Rows of a complex array as the rows of one batch item: the forward
// transform of each padded row into a spectrum buffer, then the derivative
// factor and the inverse transform, stored from column out_off on. Rows
// row0 .. row0 + nrows - 1 of A per call (the spectrum buffer holds nrows).
template <typename TC>
struct RowFftOp {
  static constexpr int NARR = 1;
  static constexpr bool kDirect = true;
  static constexpr bool kBatch = false;
  const TC* A;      // (rows, M)
  double2* xh;      // (nrows, Npad)
  int M, Npad, n1, padtype, row0, nrows;
  __device__ RowFftOp bind(int) const { return *this; }
  __device__ int rows() const { return nrows; }
  __device__ void load(int, int row, int k, double2 (&v)[1]) const {
    const int s = pad_src((long long)k - n1, M, padtype);
    if (s >= 0) {
      const TC a = A[(size_t)(row0 + row) * M + s];
      v[0] = make_double2((double)a.x, (double)a.y);
    } else {
      v[0] = make_double2(0.0, 0.0);
    }
  }
  __device__ void store(int, int row, int n, double2 (&v)[1]) const {
    xh[(size_t)row * Npad + n] = v[0];
  }
};

template <typename OC>
struct RowDiffOp {
  static constexpr int NARR = 1;
  static constexpr bool kDirect = true;
  static constexpr bool kBatch = false;
  const double2* xh;  // (nrows, Npad)
  OC* out;            // (rows, N_out)
  int Npad, row0, nrows, out_off, N_out;
  double h_fs;        // 2 pi / Npad * fs
  double inv_npad;
  __device__ RowDiffOp bind(int) const { return *this; }
  __device__ int rows() const { return nrows; }
  __device__ void load(int, int row, int k, double2 (&v)[1]) const {
    // xi_k = k h (k <= Npad/2), (k - Npad) h otherwise (wavelets.py:473-484,
    // no Nyquist halving here)
    const int kk = (k <= (Npad >> 1)) ? k : k - Npad;
    const double c = (double)kk * h_fs;
    const double2 z = xh[(size_t)row * Npad + k];
    v[0] = make_double2(-z.y * c, z.x * c);
  }
  __device__ void store(int, int row, int n, double2 (&v)[1]) const {
    const int j = n - out_off;
    if (j < 0 || j >= N_out) return;
    out[(size_t)(row0 + row) * N_out + j] =
        out_c<OC>(make_double2(v[0].x * inv_npad, v[0].y * inv_npad));
  }
};

template <typename C, typename OC = C>
struct CwtOp {
  typedef typename RealOf<C>::type T;
  typedef typename RealOf<OC>::type OT;
  static constexpr int NARR = 2;
  static constexpr bool kDirect = true;
  static constexpr bool kBatch = false;
  const double2* xh;      // (B, Npad) float64
  const double* scales;   // (na)
  WavDev wav;
  BinDev bins;
  int na, N, Npad, n1;    // N, n1: output width and the padded index of its first column
  double h;               // 2*pi / Npad
  double inv_dt;
  T inv_npad;
  double gamma;
  OC* Wx;                 // (B, na, N)
  OC* dWx;                // optional
  OT* w;                  // optional phase transform
  uint16_t* idx;          // optional bin index, (B, na, idx_pitch)
  int idx_pitch;
  int* status;
  int nrun = 0;           // rows the tile passes run (0: all na); the rest go
                          // through the band-limited single pass
  __device__ CwtOp bind(int) const { return *this; }
  __device__ int rows() const { return nrun > 0 ? nrun : na; }
  // the same op for signals b0, b0+1, ... (pointers advanced by b0 signals)
  __host__ __device__ CwtOp shifted(int b0) const {
    CwtOp o = *this;
    const size_t s = (size_t)b0;
    if (o.xh) o.xh += s * Npad;
    if (o.Wx) o.Wx += s * na * N;
    if (o.dWx) o.dWx += s * na * N;
    if (o.w) o.w += s * na * N;
    if (o.idx) o.idx += s * na * idx_pitch;
    return o;
  }
  // Split load (spectrum value first, then the wavelet), and the signed bin
  // range [klo, khi] outside which psih(scale * xi) is exactly 0 (one bin of
  // margin each side; psih still applies its own band test inside).
  static constexpr bool kSplitLoad = true;
  __device__ void band_bins(int row, int& klo, int& khi) const {
    klo = -Npad;
    khi = Npad;
    if (wav.lo < wav.hi) {
      const double sh = scales[row] * h;
      const double a = floor(wav.lo / sh) - 1.0, c = ceil(wav.hi / sh) + 1.0;
      klo = (int)fmax(fmin(a, (double)Npad), -(double)Npad);
      khi = (int)fmax(fmin(c, (double)Npad), -(double)Npad);
    }
  }
  __device__ double2 raw(int b, int k, int klo, int khi) const {
    const int kk = (k <= (Npad >> 1)) ? k : k - Npad;
    return (kk >= klo && kk <= khi) ? __ldg(xh + (size_t)b * Npad + k)
                                    : make_double2(0.0, 0.0);
  }
  __device__ void load(int b, int row, int k, C (&v)[2]) const {
    finish(b, row, k, __ldg(xh + (size_t)b * Npad + k), v);
  }
  __device__ void finish(int b, int row, int k, double2 xv, C (&v)[2]) const {
    apply(k, xv, psi(row, k), v);
  }
  // psih(scale * xi_k) with the Nyquist bin halved (wavelets.py:86-95)
  __device__ double psi(int row, int k) const {
    const int kk = (k <= (Npad >> 1)) ? k : k - Npad;
    const double xi = (double)kk * h;
    double ps = psih_fp64(wav, scales[row] * xi);
    if (k == (Npad >> 1)) ps *= 0.5;
    return ps;
  }
  __device__ void apply(int k, double2 xv, double ps, C (&v)[2]) const {
    const int kk = (k <= (Npad >> 1)) ? k : k - Npad;
    const double xi = (double)kk * h;
    const double2 y = make_double2(ps * xv.x, ps * xv.y);
    const double c = xi * inv_dt;
    v[0] = to_c<C>(y);
    v[1] = to_c<C>(make_double2(-y.y * c, y.x * c));
  }
  __device__ void store(int b, int row, int n, C (&v)[2]) const {
    const int j = n - n1;
    if (j < 0 || j >= N) return;
    C Wv = v[0], dWv = v[1];
    Wv.x *= inv_npad; Wv.y *= inv_npad;
    dWv.x *= inv_npad; dWv.y *= inv_npad;
    const size_t o = ((size_t)b * na + row) * N + j;
    if (Wx) Wx[o] = out_c<OC>(Wv);
    if (dWx) dWx[o] = out_c<OC>(dWv);
    if (idx) {
      // bins from the arithmetic-precision values, before output rounding
      double wv;
      const uint16_t k = phase_bin(Wv, dWv, 0.0, false, bins, gamma, status,
                                   w ? &wv : nullptr);
      idx[((size_t)b * na + row) * idx_pitch + j] = k;
      if (w) w[o] = (OT)wv;
    } else if (w) {
      w[o] = (OT)phase_w(Wv, dWv, 0.0, false, gamma);  // no bins asked for
    }
  }
};

// ---- fused STFT (modulated framing, stft_utils.py:69-98; _stft.py:127-147)
template <typename TX, typename C, typename OC = C>
struct StftOp {
  typedef typename RealOf<C>::type T;
  typedef typename RealOf<OC>::type OT;
  static constexpr int NARR = 1;
  static constexpr bool kDirect = false;
  static constexpr bool kBatch = false;
  const TX* x;             // (B, N)
  const double* win;       // (n_fft)
  const double* dwin;      // (n_fft), already times fs
  const double* sfs;       // (n_fft/2 + 1)
  BinDev bins;
  int N, L, hop, n1, padtype, s21, modulated, nframes;
  double gamma;
  OC* Sx;                  // (B, L/2+1, nframes)
  OC* dSx;
  OT* w;
  uint16_t* idx;           // (B, L/2+1, idx_pitch)
  int idx_pitch;
  int* status;
  __device__ StftOp bind(int) const { return *this; }
  __device__ int rows() const { return nframes; }
  __device__ void load(int b, int t, int m, C (&v)[1]) const {
    const int q = modulated ? ((m + s21) & (L - 1)) : m;
    const long long p = (long long)t * hop + q;  // position in the padded signal
    const int s = pad_src(p - n1, N, padtype);
    const double xv = s >= 0 ? (double)x[(size_t)b * N + s] : 0.0;
    v[0] = to_c<C>(make_double2(xv * __ldg(win + q), xv * __ldg(dwin + q)));
  }
  template <class LY>
  __device__ void store_smem(int b, int t, int n, C* const (&buf)[1], int f) const {
    const int nrow = (L >> 1) + 1;
    if (n >= nrow) return;
    const C zk = buf[0][LY::at(f, n)];
    const C zm = buf[0][LY::at(f, (L - n) & (L - 1))];
    const T hf = (T)0.5;
    // z = a + i*b with real a (window) and b (diff window):
    // A_k = (Z_k + conj Z_{L-k}) / 2,  B_k = (Z_k - conj Z_{L-k}) / (2i)
    const C S = mk(hf * (zk.x + zm.x), hf * (zk.y - zm.y));
    const C dS = mk(hf * (zk.y + zm.y), -hf * (zk.x - zm.x));
    const size_t o = ((size_t)b * nrow + n) * nframes + t;
    if (Sx) Sx[o] = out_c<OC>(S);
    if (dSx) dSx[o] = out_c<OC>(dS);
    if (idx) {
      double wv;
      const uint16_t k = phase_bin(S, dS, __ldg(sfs + n), true, bins, gamma, status,
                                   w ? &wv : nullptr);
      idx[((size_t)b * nrow + n) * idx_pitch + t] = k;
      if (w) w[o] = (OT)wv;
    } else if (w) {
      w[o] = (OT)phase_w(S, dS, __ldg(sfs + n), true, gamma);  // no bins asked for
    }
  }
};

// ---- batches of uneven lengths (one padded length per launch) ---------------
// bind(b) turns the batch op into the single-signal op of signal b, with its
// pointers already offset (the kernels then call it with batch index 0).
template <typename TX>
struct XhatBatchOp {
  static constexpr int NARR = 1;
  static constexpr bool kDirect = true;
  static constexpr bool kBatch = true;
  const TX* x;
  double2* xh;              // (nsig, Npad)
  const SigDesc* desc;
  int Npad, padtype;
  __device__ XhatOp<TX> bind(int b) const {
    const SigDesc& d = desc[b];
    return XhatOp<TX>{x + d.x_off, xh + (size_t)b * Npad, d.N, Npad, d.n1, padtype};
  }
};

template <typename C, typename OC>
struct CwtBatchOp {
  typedef typename RealOf<C>::type T;
  static constexpr int NARR = 2;
  static constexpr bool kDirect = true;
  static constexpr bool kBatch = true;
  const double2* xh;        // (nsig, Npad)
  const SigDesc* desc;
  WavDev wav;
  int Npad;
  double h, inv_dt;
  T inv_npad;
  double gamma;
  OC* Wx;
  uint16_t* idx;
  int* status;
  int band_from = 0x7fffffff;  // rows from here take the band-limited pass
  __device__ CwtOp<C, OC> bind(int b) const {
    const SigDesc& d = desc[b];
    const BinDev bd{d.mode, d.idx1, d.flipud, d.nbins, d.p0, d.p1, d.p2, d.p3};
    CwtOp<C, OC> o{xh + (size_t)b * Npad, d.scales, wav, bd, d.na, d.N, Npad, d.n1,
                   h, inv_dt, inv_npad, gamma, Wx + d.out_off, nullptr, nullptr,
                   idx + d.idx_off, d.idx_pitch, status};
    o.nrun = d.na < band_from ? d.na : band_from;
    return o;
  }
  // the same op for signals b0, b0+1, ... (descriptors and spectra advanced)
  __host__ __device__ CwtBatchOp shifted(int b0) const {
    CwtBatchOp o = *this;
    o.desc += b0;
    o.xh += (size_t)b0 * Npad;
    return o;
  }
};

// ---- gradient of Wx for the adjoints ----------------------------------------
// Gradient of Wx at (signal b, row i, column j): the sum of the supplied
// sources (any may be absent): the direct gradient, the squeeze's gather
// c_i gTx[idx[i, j], j] and the icwt's w_i gx[j].
template <typename C>
struct AdjSources {
  typedef typename RealOf<C>::type T;
  const C* gW;              // (B, na, N) gradient of Wx
  const C* gT;              // (B, nbins, N) gradient of Tx
  const uint16_t* idx;      // (B, na, idx_pitch) bins of the forward
  int idx_pitch, nbins;
  const double* sqw;        // (na) squeeze weights
  const T* gxr;             // (B, N) gradient of the icwt output
  const double* icw;        // (na) icwt row weights
  __device__ __forceinline__ C at(int b, int na, int N, int i, int j, int* status) const {
    C acc = mk((T)0, (T)0);
    const size_t o = ((size_t)b * na + i) * N + j;
    if (gW) acc = gW[o];
    if (gT) {
      const uint16_t k = idx[((size_t)b * na + i) * idx_pitch + j];
      if (k != kNoBin) {
        if (k < nbins) {
          const C t = gT[((size_t)b * nbins + k) * N + j];
          const T c = (T)sqw[i];
          acc.x += t.x * c;
          acc.y += t.y * c;
        } else {
          set_status(status, DEV_BAD_BIN);
        }
      }
    }
    if (gxr) acc.x += gxr[(size_t)b * N + j] * (T)icw[i];
    return acc;
  }
};

}  // namespace ssqb
