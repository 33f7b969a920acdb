// Adjoints of the forward maps, for reverse-mode differentiation of
// ssq_cwt / cwt / icwt (float32 data in float32 arithmetic, float64 data in
// float64).
//
// Forward, per row i (scale s_i) of signal b:
//   Wx_i = unpad( ifft( psih(s_i xi) * fft(pad(x)) ) )
// With g_i the gradient of Wx_i (torch's convention dL/dRe + i dL/dIm) and
// psih real, the gradient of the padded signal is
//   gxp = Re( ifft( sum_i psih(s_i xi) * fft(g_i placed at columns n1..n1+N-1) ) )
// and gx[s] sums gxp over every padded position whose source sample is s
// (the transpose of the padding). The squeeze Tx[k, j] = sum_{i: idx=k}
// c_i Wx[i, j] (bins held fixed) and the one-integral icwt
// x[j] = sum_i w_i Re Wx[i, j] have the gathers
//   gWx[i, j] += c_i gTx[idx[i, j], j],   gWx[i, j] += w_i gx[j]
// as adjoints; they run either as their own kernel or inside the row loader
// of the CWT adjoint (nothing of size (na, N) is then written).
#include "tile_launch.cuh"

namespace ssqb {

// Rows [row_lo, row_lo + nrows) -> Y (B, nrows, Npad):
// psih(s_i xi_k) * fft(g_i placed at n1)[k].
template <typename C>
struct AdjRowOp {
  typedef typename RealOf<C>::type T;
  static constexpr int NARR = 1;
  static constexpr bool kDirect = true;
  static constexpr bool kBatch = false;
  // one copy of the wavelet evaluation in the store: 37.10 vs 37.43 ms for
  // the 64 x 16,384 forward + backward, same gradients
  static constexpr bool kRolledStore = true;
  AdjSources<C> src;
  const double* scales;
  WavDev wav;
  int na, N, Npad, n1, row_lo, nrows;
  double h;                 // 2 pi / Npad
  C* Y;
  int* status;
  __device__ AdjRowOp bind(int) const { return *this; }
  __device__ int rows() const { return nrows; }
  __device__ void load(int b, int row, int k, C (&v)[1]) const {
    const int j = k - n1;
    v[0] = (j >= 0 && j < N) ? src.at(b, na, N, row_lo + row, j, status) : mk((T)0, (T)0);
  }
  __device__ void store(int b, int row, int n, C (&v)[1]) const {
    const int kk = (n <= (Npad >> 1)) ? n : n - Npad;
    const double xi = (double)kk * h;
    double ps = psih_fp64(wav, scales[row_lo + row] * xi);
    if (n == (Npad >> 1)) ps *= 0.5;  // the forward's halved Nyquist bin
    const T p = (T)ps;
    Y[((size_t)b * nrows + row) * Npad + n] = mk(v[0].x * p, v[0].y * p);
  }
};

// G[b, k] (+)= sum over the chunk's rows of Y[b, r, k], rows ascending.
template <typename C>
__global__ void adj_reduce_kernel(const C* __restrict__ Y, int B, int nrows, int Npad,
                                  C* __restrict__ G, int accumulate) {
  typedef typename RealOf<C>::type T;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)B * Npad) return;
  const size_t b = i / Npad, k = i % Npad;
  const C* y = Y + b * nrows * Npad + k;
  C s = accumulate ? G[i] : mk((T)0, (T)0);
  for (int r = 0; r < nrows; ++r) s = cadd(s, y[(size_t)r * Npad]);
  G[i] = s;
}

// Real part of the inverse transform of G: yp[b, n] = Re(ifft(G[b]))[n].
template <typename C>
struct AdjInvOp {
  typedef typename RealOf<C>::type T;
  static constexpr int NARR = 1;
  static constexpr bool kDirect = true;
  static constexpr bool kBatch = false;
  const C* G;
  T* yp;
  int Npad;
  T inv_npad;
  __device__ AdjInvOp bind(int) const { return *this; }
  __device__ int rows() const { return 1; }
  __device__ void load(int b, int, int k, C (&v)[1]) const { v[0] = G[(size_t)b * Npad + k]; }
  __device__ void store(int b, int, int n, C (&v)[1]) const {
    yp[(size_t)b * Npad + n] = v[0].x * inv_npad;
  }
};

// Calls f(q) for every padded offset q in [qlo, qhi) (relative to x[0])
// whose source sample is s: q = s first, then the images of the padding's
// one or two residue families (period P), ascending.
template <class F>
__device__ __forceinline__ void for_each_image(int s, int N, long long qlo, long long qhi,
                                               int padtype, const F& f) {
  if (s >= qlo && s < qhi) f((long long)s);
  long long P = 1, a[2] = {s, s};
  int nf = 0;
  if (padtype == PAD_REFLECT && N > 1) { P = 2LL * (N - 1); a[0] = s; a[1] = -s; nf = 2; }
  else if (padtype == PAD_SYMMETRIC) { P = 2LL * N; a[0] = s; a[1] = -1 - s; nf = 2; }
  else if (padtype == PAD_WRAP) { P = N; a[0] = s; nf = 1; }
  for (int fam = 0; fam < nf; ++fam) {
    // k from ceil((qlo - a) / P) to floor((qhi - 1 - a) / P)
    const long long lo = qlo - a[fam], hi = qhi - 1 - a[fam];
    const long long k0 = lo >= 0 ? (lo + P - 1) / P : -((-lo) / P);
    for (long long k = k0; k * P <= hi; ++k) {
      const long long q = a[fam] + k * P;
      if (q >= 0 && q < N) continue;                            // the signal itself
      if (fam == 1 && ((q - a[0]) % P + P) % P == 0) continue;  // already in family 0
      if (pad_src(q, N, padtype) != s) continue;
      f(q);
    }
  }
}

// gx[b, s] (+)= sum of yp[b, n1 + q] over the padded offsets q whose source
// is s (the transpose of the padding).
template <typename T>
__global__ void adj_fold_kernel(const T* __restrict__ yp, int B, int N, int Npad, int n1,
                                int padtype, T* __restrict__ gx, int accumulate) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)B * N) return;
  const int b = (int)(i / N), s = (int)(i % N);
  const T* y = yp + (size_t)b * Npad + n1;
  T acc = 0;
  for_each_image(s, N, -(long long)n1, (long long)Npad - n1, padtype,
                 [&](long long q) { acc += y[q]; });
  gx[i] = accumulate ? gx[i] + acc : acc;
}

// ---- STFT adjoint ------------------------------------------------------------
// Forward: frame t, element m, u[t, m] = xp[t hop + q(m)] win[q(m)] with
// q(m) = (m + s21) mod L (modulated) or m; Sx[f, t] = sum_m u[t, m] e^{-2 pi i f m / L}
// for f <= L/2. Adjoint: gu[t, m] = Re sum_{f <= L/2} g[f, t] e^{+2 pi i f m / L},
// then gx[s] = sum over the frames and elements reading s of win[q] gu[t, m].
template <typename C>
struct StftAdjOp {
  typedef typename RealOf<C>::type T;
  static constexpr int NARR = 1;
  static constexpr bool kDirect = false;
  static constexpr bool kBatch = false;
  static constexpr int kMapIn = MAP_F;  // consecutive threads: consecutive frames
  AdjSources<C> src;                    // gradient of Sx (B, nrow, nframes)
  int L, nrow, nframes;
  T* gu;                                // (B, L, nframes), element-major
  int* status;
  int interior2;                        // 1: bins 0 < f < L/2 doubled (inverse rfft)
  __device__ StftAdjOp bind(int) const { return *this; }
  __device__ int rows() const { return nframes; }
  __device__ void load(int b, int t, int f, C (&v)[1]) const {
    v[0] = f < nrow ? src.at(b, nrow, nframes, f, t, status) : mk((T)0, (T)0);
    if (interior2 && f > 0 && f < L / 2) {
      v[0].x *= (T)2;
      v[0].y *= (T)2;
    }
  }
  template <class LY>
  __device__ void store_smem(int b, int t, int n, C* const (&buf)[1], int fr) const {
    gu[((size_t)b * L + n) * nframes + t] = buf[0][LY::at(fr, n)].x;
  }
};

template <typename T>
__global__ void stft_adj_gather_kernel(const T* __restrict__ gu, const double* __restrict__ win,
                                       int B, int N, int L, int hop, int nframes, int n1,
                                       int padtype, int modulated, int s21,
                                       T* __restrict__ gx, int accumulate) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)B * N) return;
  const int b = (int)(i / N), s = (int)(i % N);
  const T* g = gu + (size_t)b * L * nframes;
  const long long ptot = (long long)(nframes - 1) * hop + L;  // padded positions read
  T acc = 0;
  for_each_image(s, N, -(long long)n1, ptot - n1, padtype, [&](long long qq) {
    const long long p = qq + n1;
    const long long num = p - L + 1;
    const long long tlo = num <= 0 ? 0 : (num + hop - 1) / hop;
    long long thi = p / hop;
    if (thi > nframes - 1) thi = nframes - 1;
    for (long long t = thi; t >= tlo; --t) {
      const int q = (int)(p - t * hop);
      const int m = modulated ? ((q - s21) % L + L) % L : q;
      acc += (T)__ldg(win + q) * g[(size_t)m * nframes + t];
    }
  });
  gx[i] = accumulate ? gx[i] + acc : acc;
}

// ---- inverse STFT (_stft.py:184-256, utils/stft_utils.py:141-191) ------------
// Frame t of the inverse is xbuf[m, t] = irfft(Sx[:, t])[m]
//   = (1/L) Re sum_{f <= L/2} c_f Sx[f, t] e^{+2 pi i f m / L},
// c_0 = c_{L/2} = 1, c_f = 2 otherwise (the imaginary parts of the DC and
// Nyquist bins drop out of the real part): StftAdjOp with the interior bins
// doubled, 1/L applied here (a power of two, so exact). A modulated frame is
// fftshifted, for even L a rotation by L/2. Overlap-add with wa = window^a
// over frames in ascending order, as the reference does, then divide by the
// window norm wn[p] = sum_{t < maxhops} w1[p - t hop], w1 = window^(a+1),
// where wn > tiny (the reference divides everywhere when min(wn) >= tiny and
// only where wn > tiny otherwise; the two differ only where wn == tiny).
// Output: the padded positions p = L/2 .. L/2 + N - 1 the reference keeps.
// Sums run in double for either data precision.
template <typename T>
__global__ void istft_ola_kernel(const T* __restrict__ gu, const double* __restrict__ wa,
                                 const double* __restrict__ w1, int B, int N, int L, int hop,
                                 int nframes, int maxhops, int modulated, double tiny,
                                 T* __restrict__ x) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)B * N) return;
  const int b = (int)(i / N), s = (int)(i % N);
  const T* g = gu + (size_t)b * L * nframes;
  const int half = L / 2;
  const int shift = (L + 1) / 2;  // fftshift: frame index m of padded offset q
  const long long p = (long long)s + half;
  const long long num = p - L + 1;
  const long long tlo = num <= 0 ? 0 : (num + hop - 1) / hop;
  const long long tmax = p / hop;
  const long long thi = tmax < nframes - 1 ? tmax : nframes - 1;
  const long long tw = tmax < maxhops - 1 ? tmax : maxhops - 1;
  double acc = 0.0, wn = 0.0;
  for (long long t = tlo; t <= thi; ++t) {
    const int q = (int)(p - t * hop);
    const int m = modulated ? (q + shift) % L : q;
    acc += (double)g[(size_t)m * nframes + t] * wa[q];
  }
  for (long long t = tlo; t <= tw; ++t) wn += w1[(int)(p - t * hop)];
  acc *= 1.0 / L;
  x[i] = (T)(wn > tiny ? acc / wn : acc);
}

template <typename C>
static int run_istft(const C* Sx, int B, int N, int L, int hop, int nframes, int modulated,
                     const double* wa, const double* w1, double tiny,
                     typename RealOf<C>::type* x, void* ws, const Tables& tb,
                     cudaStream_t st) {
  typedef typename RealOf<C>::type T;
  const int nrow = L / 2 + 1;
  int e;
  if (L & (L - 1)) {  // not a power of two: frames by the chirp-z kernel
    if constexpr (std::is_same<C, double2>::value)
      e = run_istft_frames_any_f64(Sx, B, L, nframes, (double*)ws, tb, st);
    else
      e = run_istft_frames_any_f32(Sx, B, L, nframes, (float*)ws, tb, st);
    if (e) return e;
    if (int* c = launch_counter()) return ++*c, 0;
  } else {
    AdjSources<C> src{Sx, nullptr, nullptr, 0, nrow, nullptr, nullptr, nullptr};
    StftAdjOp<C> op{src, L, nrow, nframes, (T*)ws, tb.status, 1};
    e = run_single<StftAdjOp<C>, C, 1>(op, B, nframes, ilog2(L), tb, st);
    if (e) return e;
  }
  if (int* c = launch_counter()) return ++*c, 0;
  const int maxhops = (N - 1) / hop + 1;
  const size_t n = (size_t)B * N;
  istft_ola_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
      (const T*)ws, wa, w1, B, N, L, hop, nframes, maxhops, modulated, tiny, x);
  return cudaGetLastError();
}

int run_istft_f32(const float2* Sx, int B, int N, int L, int hop, int nframes, int modulated,
                  const double* wa, const double* w1, double tiny, float* x, void* ws,
                  const Tables& tb, cudaStream_t st) {
  return run_istft<float2>(Sx, B, N, L, hop, nframes, modulated, wa, w1, tiny, x, ws, tb, st);
}

int run_istft_f64(const double2* Sx, int B, int N, int L, int hop, int nframes, int modulated,
                  const double* wa, const double* w1, double tiny, double* x, void* ws,
                  const Tables& tb, cudaStream_t st) {
  return run_istft<double2>(Sx, B, N, L, hop, nframes, modulated, wa, w1, tiny, x, ws, tb, st);
}

template <typename C>
__global__ void wx_adj_kernel(AdjSources<C> src, int B, int na, int N, C* __restrict__ gWx,
                              int accumulate, int* status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const int i = blockIdx.y, b = blockIdx.z;
  const C v = src.at(b, na, N, i, j, status);
  const size_t o = ((size_t)b * na + i) * N + j;
  gWx[o] = accumulate ? cadd(gWx[o], v) : v;
}

// ---- host side ---------------------------------------------------------------

static size_t adj_row_bytes(int B, int Npad, size_t cs) {
  return (size_t)2 * B * Npad * cs;  // Y + Z of one row
}

size_t cwt_adjoint_workspace(int B, int Npad, int na, bool f64) {
  const size_t cs = f64 ? sizeof(double2) : sizeof(float2);
  const size_t rs = f64 ? sizeof(double) : sizeof(float);
  const size_t per_row = adj_row_bytes(B, Npad, cs);
  size_t rows = kAdjChunkBytes / per_row;
  if (rows < 1) rows = 1;
  if (rows > (size_t)na) rows = na;
  // the chunk also holds the intermediate of the final inverse (B Npad)
  return (size_t)B * Npad * cs + (size_t)B * Npad * rs + rows * per_row;
}

template <typename C>
static int run_adjoint(const AdjSources<C>& src, int B, int N, int Npad, int n1, int padtype,
                       const double* scales, int na, const WavDev& wd,
                       typename RealOf<C>::type* gx, int accumulate, void* ws,
                       size_t ws_bytes, const Tables& tb, cudaStream_t st) {
  typedef typename RealOf<C>::type T;
  const size_t cs = sizeof(C);
  C* G = (C*)ws;
  T* yp = (T*)((unsigned char*)ws + (size_t)B * Npad * cs);
  unsigned char* rest = (unsigned char*)yp + (size_t)B * Npad * sizeof(T);
  const size_t used = (size_t)(rest - (unsigned char*)ws);
  if (ws_bytes < used) return (int)cudaErrorInvalidValue;
  const size_t rest_bytes = ws_bytes - used;
  const size_t per_row = adj_row_bytes(B, Npad, cs);
  int S = (int)((rest_bytes / per_row) < (size_t)na ? rest_bytes / per_row : (size_t)na);
  if (S < 1) return (int)cudaErrorInvalidValue;
  C* Y = (C*)rest;
  C* Z = Y + (size_t)B * S * Npad;
  const int m = ilog2(Npad);
  const int nt = 256;
  for (int r0 = 0; r0 < na; r0 += S) {
    const int rows = (na - r0) < S ? (na - r0) : S;
    AdjRowOp<C> op{src, scales, wd, na, N, Npad, n1, r0, rows, (2 * M_PI) / Npad, Y,
                   tb.status};
    int e = run_tile<AdjRowOp<C>, C, -1>(op, B, rows, m, Z, (size_t)B * rows * Npad, tb, st);
    if (e) return e;
    if (int* c = launch_counter()) {
      ++*c;
    } else {
      const size_t n = (size_t)B * Npad;
      adj_reduce_kernel<C><<<(unsigned)((n + nt - 1) / nt), nt, 0, st>>>(Y, B, rows, Npad, G,
                                                                          r0 > 0);
      if ((e = cudaGetLastError())) return e;
    }
  }
  AdjInvOp<C> inv{G, yp, Npad, (T)(1.0 / Npad)};
  int e = run_tile<AdjInvOp<C>, C, 1>(inv, B, 1, m, Y, rest_bytes / cs, tb, st);
  if (e) return e;
  if (int* c = launch_counter()) {
    ++*c;
    return 0;
  }
  const size_t n = (size_t)B * N;
  adj_fold_kernel<T><<<(unsigned)((n + nt - 1) / nt), nt, 0, st>>>(yp, B, N, Npad, n1, padtype,
                                                                    gx, accumulate);
  return cudaGetLastError();
}

template <typename C>
static int run_stft_adj(const AdjSources<C>& src, int B, int N, int L, int hop, int n1,
                        int padtype, int modulated, const double* win,
                        typename RealOf<C>::type* gx, int accumulate, void* ws,
                        const Tables& tb, cudaStream_t st) {
  typedef typename RealOf<C>::type T;
  const int nframes = (N - 1) / hop + 1;
  int e;
  if (L & (L - 1)) {  // not a power of two: the chirp-z frame transform
    if constexpr (std::is_same<C, double2>::value)
      e = run_adj_frames_any_f64(src, B, L, nframes, (double*)ws, tb, st);
    else
      e = run_adj_frames_any_f32(src, B, L, nframes, (float*)ws, tb, st);
  } else {
    StftAdjOp<C> op{src, L, L / 2 + 1, nframes, (T*)ws, tb.status, 0};
    e = run_single<StftAdjOp<C>, C, 1>(op, B, nframes, ilog2(L), tb, st);
  }
  if (e) return e;
  if (int* c = launch_counter()) return ++*c, 0;
  const int s20 = (L + 1) / 2;
  const int s21 = (L % 2 == 1) ? s20 - 1 : s20;
  const size_t n = (size_t)B * N;
  stft_adj_gather_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
      (const T*)ws, win, B, N, L, hop, nframes, n1, padtype, modulated, s21, gx, accumulate);
  return cudaGetLastError();
}

int run_stft_adjoint_f32(const AdjSources<float2>& src, int B, int N, int L, int hop, int n1,
                         int padtype, int modulated, const double* win, float* gx,
                         int accumulate, void* ws, const Tables& tb, cudaStream_t st) {
  return run_stft_adj<float2>(src, B, N, L, hop, n1, padtype, modulated, win, gx, accumulate,
                              ws, tb, st);
}

int run_stft_adjoint_f64(const AdjSources<double2>& src, int B, int N, int L, int hop, int n1,
                         int padtype, int modulated, const double* win, double* gx,
                         int accumulate, void* ws, const Tables& tb, cudaStream_t st) {
  return run_stft_adj<double2>(src, B, N, L, hop, n1, padtype, modulated, win, gx, accumulate,
                               ws, tb, st);
}

int run_cwt_adjoint_f32(const AdjSources<float2>& src, int B, int N, int Npad, int n1,
                        int padtype, const double* scales, int na, const WavDev& wd, float* gx,
                        int accumulate, void* ws, size_t ws_bytes, const Tables& tb,
                        cudaStream_t st) {
  return run_adjoint<float2>(src, B, N, Npad, n1, padtype, scales, na, wd, gx, accumulate, ws,
                             ws_bytes, tb, st);
}

int run_cwt_adjoint_f64(const AdjSources<double2>& src, int B, int N, int Npad, int n1,
                        int padtype, const double* scales, int na, const WavDev& wd,
                        double* gx, int accumulate, void* ws, size_t ws_bytes,
                        const Tables& tb, cudaStream_t st) {
  return run_adjoint<double2>(src, B, N, Npad, n1, padtype, scales, na, wd, gx, accumulate,
                              ws, ws_bytes, tb, st);
}

template <typename C>
static int run_wx_adj(const AdjSources<C>& src, int B, int na, int N, C* gWx, int accumulate,
                      int* status, cudaStream_t st) {
  if (int* c = launch_counter()) return ++*c, 0;
  dim3 grid((N + 255) / 256, na, B);
  wx_adj_kernel<C><<<grid, 256, 0, st>>>(src, B, na, N, gWx, accumulate, status);
  return cudaGetLastError();
}

int run_wx_adjoint_f32(const AdjSources<float2>& src, int B, int na, int N, float2* gWx,
                       int accumulate, int* status, cudaStream_t st) {
  return run_wx_adj<float2>(src, B, na, N, gWx, accumulate, status, st);
}

int run_wx_adjoint_f64(const AdjSources<double2>& src, int B, int na, int N, double2* gWx,
                       int accumulate, int* status, cudaStream_t st) {
  return run_wx_adj<double2>(src, B, na, N, gWx, accumulate, status, st);
}

}  // namespace ssqb
