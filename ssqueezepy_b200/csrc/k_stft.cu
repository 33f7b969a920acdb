// Fused STFT tile kernels (one pass; power-of-two n_fft up to one tile).
#include "tile_launch.cuh"
#include "fft_mixed.cuh"

namespace ssqb {

template <class Op, typename C, int LOGL>
static int launch_stft(const Op& op, int B, const Tables& tb, cudaStream_t st) {
  constexpr int NF = tile_of<C>() / (1 << LOGL);
  const size_t smem = tile_smem<C>(Op::NARR, LOGL);
  auto k = tile_single<Op, C, LOGL, -1>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  dim3 grid((op.nframes + NF - 1) / NF, 1, B);
  k<<<grid, kNT, smem, st>>>(op, tb);
  return cudaGetLastError();
}

template <class Op, typename C>
static int run_stft(const Op& op, int B, int log2L, const Tables& tb, cudaStream_t st) {
  return dispatch_log<3, tile_log<C>()>(log2L, [&](auto k) {
    return launch_stft<Op, C, decltype(k)::value>(op, B, tb, st);
  });
}

// ---- any n_fft: Bluestein's chirp-z transform in one kernel -------------------
// With c_n = e^{-i pi n^2 / L}, the length-L DFT of a frame is
//   Z_k = c_k (a (*) b)_k,  a_m = z_m c_m (m < L, zero up to M),
//   b_n = conj(c_n) for n and M - n, 0 <= n < L (zero between),
// a circular convolution of power-of-two length M >= 2L - 1, so three
// tile FFTs of M per frame: b's transform, a's transform, and the inverse of
// their product, all in shared memory; then the Hermitian split of the
// window / derivative-window pair and the phase / bin epilogue of StftOp.
// Arithmetic in float64 for every data precision; M <= the float64 tile.
__device__ __forceinline__ double2 chirp(int n, int L) {
  // n^2 mod 2L keeps the angle exact before the trigonometric call
  const long long r = ((long long)n * n) % (2LL * L);
  double sv, cv;
  sincospi((double)r / (double)L, &sv, &cv);
  return make_double2(cv, -sv);
}

struct NoStore {
  template <int R>
  __device__ void item(int, int, int, double2 (&)[R], double2 (&)[R]) const {}
};

// Two CTAs per SM (128 registers, a few hundred bytes spilled) instead of one
// at 204-214 registers, for both chirp-z kernels. At N = 160,000: ssq_stft
// 1.33x at n_fft 598 and 1000, 1.45x at 121; istft 1.18x, 1.47x, 1.19x.
constexpr int kBluesteinCtas = 2;

template <typename TX, typename OC, int LOGM>
__global__ void __launch_bounds__(kNT, kBluesteinCtas)
stft_bluestein_kernel(StftOp<TX, double2, OC> op, Tables tb) {
  typedef double2 C;
  typedef typename RealOf<OC>::type OT;
  constexpr int M = 1 << LOGM;
  constexpr int NF = tile_of<C>() / M;
  typedef Layout<C, LOGM, NF> LY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* const bufA[1] = {base};
  C* const bufB[1] = {base + LY::ARR};
  C* const bufC[1] = {base + 2 * LY::ARR};
  const int b = blockIdx.z;
  const int L = op.L;
  const C zero = make_double2(0.0, 0.0);
  const NoStore st{};
  // b's transform, the same for every frame: once per CTA, which then walks
  // the tiles of frames blockIdx.x, blockIdx.x + gridDim.x, ...
  auto ldB = [&](int, int m, C (&v)[1]) {
    v[0] = m < L ? chirp(m, L) : (m > M - L ? chirp(M - m, L) : zero);
    v[0].y = -v[0].y;  // conj(c)
  };
  fft_rows<C, LOGM, NF, kNT, -1, 1, MAP_J, MAP_J, false>(bufB, seg_table<C>(tb), ldB, st);
  const int ntile = (op.nframes + NF - 1) / NF;
  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
  const int t0 = tile * NF;
  // a's transform: the windowed frame times the chirp
  auto ldA = [&](int f, int m, C (&v)[1]) {
    const int t = t0 + f;
    if (t >= op.nframes || m >= L) {
      v[0] = zero;
      return;
    }
    const int q = op.modulated ? (m + op.s21) % L : m;
    const long long p = (long long)t * op.hop + q;
    const int s = pad_src(p - op.n1, op.N, op.padtype);
    const double xv = s >= 0 ? (double)op.x[(size_t)b * op.N + s] : 0.0;
    const C z = make_double2(xv * __ldg(op.win + q), xv * __ldg(op.dwin + q));
    v[0] = cmul(z, chirp(m, L));
  };
  fft_rows<C, LOGM, NF, kNT, -1, 1, MAP_J, MAP_J, false>(bufA, seg_table<C>(tb), ldA, st);
  // inverse transform of the product
  auto ldC = [&](int f, int m, C (&v)[1]) {
    v[0] = cmul(bufA[0][LY::at(f, m)], bufB[0][LY::at(f, m)]);
  };
  fft_rows<C, LOGM, NF, kNT, 1, 1, MAP_J, MAP_J, false>(bufC, seg_table<C>(tb), ldC, st);
  const int nrow = (L >> 1) + 1;
  const double inv_m = 1.0 / M;
  for (int e = threadIdx.x; e < NF * nrow; e += kNT) {
    const int f = e % NF, n = e / NF;
    const int t = t0 + f;
    if (t >= op.nframes) continue;
    const int nm = (L - n) % L;
    C zk = cmul(bufC[0][LY::at(f, n)], chirp(n, L));
    C zm = cmul(bufC[0][LY::at(f, nm)], chirp(nm, L));
    zk.x *= inv_m; zk.y *= inv_m;
    zm.x *= inv_m; zm.y *= inv_m;
    const double hf = 0.5;
    const C S = make_double2(hf * (zk.x + zm.x), hf * (zk.y - zm.y));
    const C dS = make_double2(hf * (zk.y + zm.y), -hf * (zk.x - zm.x));
    const size_t o = ((size_t)b * nrow + n) * op.nframes + t;
    if (op.Sx) op.Sx[o] = out_c<OC>(S);
    if (op.dSx) op.dSx[o] = out_c<OC>(dS);
    if (op.idx) {
      double wv;
      const uint16_t k = phase_bin(S, dS, __ldg(op.sfs + n), true, op.bins, op.gamma,
                                   op.status, op.w ? &wv : nullptr);
      op.idx[((size_t)b * nrow + n) * op.idx_pitch + t] = k;
      if (op.w) op.w[o] = (OT)wv;
    } else if (op.w) {
      op.w[o] = (OT)phase_w(S, dS, __ldg(op.sfs + n), true, op.gamma);
    }
  }
  __syncthreads();  // bufC is rewritten by the next tile
  }
}

template <typename TX, typename OC, int LOGM>
static int launch_bluestein(const StftOp<TX, double2, OC>& op, int B, const Tables& tb,
                            cudaStream_t st) {
  constexpr int NF = tile_of<double2>() / (1 << LOGM);
  const size_t smem = 3 * tile_smem<double2>(1, LOGM);
  auto k = stft_bluestein_kernel<TX, OC, LOGM>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  // persistent CTAs: as many as are resident (at most one per tile of frames)
  int dev = 0, sms = 148, per_sm = 1;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kNT, smem) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
    per_sm = 1;
  }
  const int ntile = (op.nframes + NF - 1) / NF;
  int gx = sms * (per_sm > 0 ? per_sm : 1);
  if (B > 1) gx = (gx + B - 1) / B;
  if (gx > ntile) gx = ntile;
  dim3 grid(gx, 1, B);
  k<<<grid, kNT, smem, st>>>(op, tb);
  return cudaGetLastError();
}

// The same chirp-z transform with a convolution length M = 3 * 2^k or 5 * 2^k
// (mixed-radix Stockham, fft_mixed.cuh) where that is shorter than the power
// of two: n_fft 598 convolves at 1280 instead of 2048. The twiddle table
// W[m] = exp(2 pi i m / M) (at tw_pos(m)) is filled once per (persistent) CTA.
// 320 threads: the radix-4 stages of 1280 = 5 x 4^4 have 320 items each
// (measured at n_fft 598: 7.30 ms per N=160,000 ssq_stft against 7.72 at the
// power of two 2048; 256 threads with 5 x 8 x 8 x 4: 9.40, 160 threads:
// 8.24; 1536 = 3 x 8^3 for n_fft 700: 11.5 against 8.2 at 2048, not used)
constexpr int kBluNT = 320;
typedef Radices<5, 4, 4, 4, 4> Radices1280;

template <typename TX, typename OC, int M, class RL>
__global__ void __launch_bounds__(kBluNT, kBluesteinCtas)
stft_bluestein_mixed_kernel(StftOp<TX, double2, OC> op, Tables tb) {
  typedef double2 C;
  typedef typename RealOf<OC>::type OT;
  constexpr int NF = tile_of<C>() / M;
  typedef LayoutM<C, M, NF> LY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const bufA = reinterpret_cast<C*>(smem_raw);
  C* const bufB = bufA + LY::ARR;
  C* const bufC = bufA + 2 * LY::ARR;
  C* const W = bufA + 3 * LY::ARR;
  const int b = blockIdx.z;
  const int L = op.L;
  const C zero = make_double2(0.0, 0.0);
  for (int m = threadIdx.x; m < M; m += kBluNT) {
    double sv, cv;
    sincospi((double)(2 * m) / (double)M, &sv, &cv);
    W[tw_pos(m)] = make_double2(cv, sv);
  }
  __syncthreads();
  auto ldB = [&](int, int m, C (&v)[1]) {
    v[0] = m < L ? chirp(m, L) : (m > M - L ? chirp(M - m, L) : zero);
    v[0].y = -v[0].y;  // conj(c)
  };
  fft_mixed_rows<C, M, NF, kBluNT, -1, RL>(bufB, W, ldB);
  const int ntile = (op.nframes + NF - 1) / NF;
  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int t0 = tile * NF;
    auto ldA = [&](int f, int m, C (&v)[1]) {
      const int t = t0 + f;
      if (t >= op.nframes || m >= L) {
        v[0] = zero;
        return;
      }
      const int q = op.modulated ? (m + op.s21) % L : m;
      const long long p = (long long)t * op.hop + q;
      const int s = pad_src(p - op.n1, op.N, op.padtype);
      const double xv = s >= 0 ? (double)op.x[(size_t)b * op.N + s] : 0.0;
      const C z = make_double2(xv * __ldg(op.win + q), xv * __ldg(op.dwin + q));
      v[0] = cmul(z, chirp(m, L));
    };
    fft_mixed_rows<C, M, NF, kBluNT, -1, RL>(bufA, W, ldA);
    auto ldC = [&](int f, int m, C (&v)[1]) {
      v[0] = cmul(bufA[LY::at(f, m)], bufB[LY::at(f, m)]);
    };
    fft_mixed_rows<C, M, NF, kBluNT, 1, RL>(bufC, W, ldC);
    const int nrow = (L >> 1) + 1;
    const double inv_m = 1.0 / M;
    for (int e = threadIdx.x; e < NF * nrow; e += kBluNT) {
      const int f = e % NF, n = e / NF;
      const int t = t0 + f;
      if (t >= op.nframes) continue;
      const int nm = (L - n) % L;
      C zk = cmul(bufC[LY::at(f, n)], chirp(n, L));
      C zm = cmul(bufC[LY::at(f, nm)], chirp(nm, L));
      zk.x *= inv_m; zk.y *= inv_m;
      zm.x *= inv_m; zm.y *= inv_m;
      const double hf = 0.5;
      const C S = make_double2(hf * (zk.x + zm.x), hf * (zk.y - zm.y));
      const C dS = make_double2(hf * (zk.y + zm.y), -hf * (zk.x - zm.x));
      const size_t o = ((size_t)b * nrow + n) * op.nframes + t;
      if (op.Sx) op.Sx[o] = out_c<OC>(S);
      if (op.dSx) op.dSx[o] = out_c<OC>(dS);
      if (op.idx) {
        double wv;
        const uint16_t k = phase_bin(S, dS, __ldg(op.sfs + n), true, op.bins, op.gamma,
                                     op.status, op.w ? &wv : nullptr);
        op.idx[((size_t)b * nrow + n) * op.idx_pitch + t] = k;
        if (op.w) op.w[o] = (OT)wv;
      } else if (op.w) {
        op.w[o] = (OT)phase_w(S, dS, __ldg(op.sfs + n), true, op.gamma);
      }
    }
    __syncthreads();  // bufC is rewritten by the next tile
  }
}

template <typename TX, typename OC, int M, class RL>
static int launch_bluestein_mixed(const StftOp<TX, double2, OC>& op, int B, const Tables& tb,
                                  cudaStream_t st) {
  constexpr int NF = tile_of<double2>() / M;
  typedef LayoutM<double2, M, NF> LY;
  const size_t smem = (3 * (size_t)LY::ARR + M) * sizeof(double2);
  auto k = stft_bluestein_mixed_kernel<TX, OC, M, RL>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  int dev = 0, sms = 148, per_sm = 1;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kBluNT, smem) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
    per_sm = 1;
  }
  const int ntile = (op.nframes + NF - 1) / NF;
  int gx = sms * (per_sm > 0 ? per_sm : 1);
  if (B > 1) gx = (gx + B - 1) / B;
  if (gx > ntile) gx = ntile;
  dim3 grid(gx, 1, B);
  k<<<grid, kBluNT, smem, st>>>(op, tb);
  return cudaGetLastError();
}

// Convolution length of the chirp-z transform of an n_fft of L: 1280 where
// that suffices and the power of two would be 2048 (n_fft 513-640), else the
// smallest power of two >= 2L - 1.
static int bluestein_length(int L) {
  int m = 8;
  while (m < 2 * L - 1) m *= 2;
  return (m == 2048 && 2 * L - 1 <= 1280) ? 1280 : m;
}

template <typename TX, typename OC>
static int run_bluestein(const StftOp<TX, double2, OC>& op, int B, int log2M,
                         const Tables& tb, cudaStream_t st) {
  switch (bluestein_length(op.L)) {
    case 1280: return launch_bluestein_mixed<TX, OC, 1280, Radices1280>(op, B, tb, st);
    default:
      return dispatch_log<3, tile_log<double2>()>(log2M, [&](auto k) {
        return launch_bluestein<TX, OC, decltype(k)::value>(op, B, tb, st);
      });
  }
}

// ---- istft frames for any n_fft: the inverse real transform by chirp-z ------
// y_m = sum_k X_k e^{+2 pi i k m / L} = conj(c_m) (a' (*) c)_m with
// a'_k = X_k conj(c_k), X_k = c_k' S_k for k <= L/2 (c_k' = 1 at k = 0 and
// k = L/2, else 2: the one-sided spectrum of a real frame), 0 above; the
// frame is Re y (1/L is applied by the overlap-add). Frames go to gu
// (B, L, nframes), element-major, as the power-of-two path writes them.
// One-sided inputs of the frame transform: the spectrum of istft (interior
// bins doubled), or the gradient sources of the STFT adjoint (weights 1).
template <typename CI>
struct SpecSrc {
  const CI* Sx;
  __device__ double2 at(int b, int nrow, int nframes, int k, int t, int L) const {
    const CI sv = Sx[((size_t)b * nrow + k) * nframes + t];
    const double wk = (k == 0 || 2 * k == L) ? 1.0 : 2.0;
    return make_double2(wk * (double)sv.x, wk * (double)sv.y);
  }
};
template <typename CI>
struct AdjSrc {
  AdjSources<CI> src;
  int* status;
  __device__ double2 at(int b, int nrow, int nframes, int k, int t, int) const {
    const CI v = src.at(b, nrow, nframes, k, t, status);
    return make_double2((double)v.x, (double)v.y);
  }
};

template <class Src, typename T, int LOGM>
__global__ void __launch_bounds__(kNT, kBluesteinCtas)
istft_frames_bluestein_kernel(Src src, int L, int nframes, T* __restrict__ gu, Tables tb) {
  typedef double2 C;
  constexpr int M = 1 << LOGM;
  constexpr int NF = tile_of<C>() / M;
  typedef Layout<C, LOGM, NF> LY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* const bufA[1] = {base};
  C* const bufB[1] = {base + LY::ARR};
  C* const bufC[1] = {base + 2 * LY::ARR};
  const int b = blockIdx.z;
  const int nrow = L / 2 + 1;
  const C zero = make_double2(0.0, 0.0);
  const NoStore st{};
  auto ldB = [&](int, int m, C (&v)[1]) {
    v[0] = m < L ? chirp(m, L) : (m > M - L ? chirp(M - m, L) : zero);
  };
  fft_rows<C, LOGM, NF, kNT, -1, 1, MAP_J, MAP_J, false>(bufB, seg_table<C>(tb), ldB, st);
  const int ntile = (nframes + NF - 1) / NF;
  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int t0 = tile * NF;
    auto ldA = [&](int f, int k, C (&v)[1]) {
      const int t = t0 + f;
      if (t >= nframes || k >= nrow) {
        v[0] = zero;
        return;
      }
      C c = chirp(k, L);
      c.y = -c.y;
      v[0] = cmul(src.at(b, nrow, nframes, k, t, L), c);
    };
    fft_rows<C, LOGM, NF, kNT, -1, 1, MAP_J, MAP_J, false>(bufA, seg_table<C>(tb), ldA, st);
    auto ldC = [&](int f, int m, C (&v)[1]) {
      v[0] = cmul(bufA[0][LY::at(f, m)], bufB[0][LY::at(f, m)]);
    };
    fft_rows<C, LOGM, NF, kNT, 1, 1, MAP_J, MAP_J, false>(bufC, seg_table<C>(tb), ldC, st);
    for (int e = threadIdx.x; e < NF * L; e += kNT) {
      const int f = e % NF, m = e / NF;
      const int t = t0 + f;
      if (t >= nframes) continue;
      C c = chirp(m, L);
      c.y = -c.y;
      const C y = cmul(bufC[0][LY::at(f, m)], c);
      gu[((size_t)b * L + m) * nframes + t] = (T)(y.x / M);
    }
    __syncthreads();  // bufA / bufC are rewritten by the next tile
  }
}

template <class Src, typename T, int LOGM>
static int launch_istft_frames(const Src& src, int B, int L, int nframes, T* gu,
                               const Tables& tb, cudaStream_t st) {
  constexpr int NF = tile_of<double2>() / (1 << LOGM);
  const size_t smem = 3 * tile_smem<double2>(1, LOGM);
  auto k = istft_frames_bluestein_kernel<Src, T, LOGM>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  int dev = 0, sms = 148, per_sm = 1;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kNT, smem) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
    per_sm = 1;
  }
  const int ntile = (nframes + NF - 1) / NF;
  int gx = sms * (per_sm > 0 ? per_sm : 1);
  if (B > 1) gx = (gx + B - 1) / B;
  if (gx > ntile) gx = ntile;
  k<<<dim3(gx, 1, B), kNT, smem, st>>>(src, L, nframes, gu, tb);
  return cudaGetLastError();
}

template <class Src, typename T>
static int run_frames_any(const Src& src, int B, int L, int nframes, T* gu, const Tables& tb,
                          cudaStream_t st) {
  int log2M = 0;
  while ((1 << log2M) < 2 * L - 1) ++log2M;
  return dispatch_log<3, tile_log<double2>()>(log2M, [&](auto k) {
    return launch_istft_frames<Src, T, decltype(k)::value>(src, B, L, nframes, gu, tb, st);
  });
}

int run_istft_frames_any_f32(const float2* Sx, int B, int L, int nframes, float* gu,
                             const Tables& tb, cudaStream_t st) {
  return run_frames_any(SpecSrc<float2>{Sx}, B, L, nframes, gu, tb, st);
}

int run_istft_frames_any_f64(const double2* Sx, int B, int L, int nframes, double* gu,
                             const Tables& tb, cudaStream_t st) {
  return run_frames_any(SpecSrc<double2>{Sx}, B, L, nframes, gu, tb, st);
}

int run_adj_frames_any_f32(const AdjSources<float2>& src, int B, int L, int nframes,
                           float* gu, const Tables& tb, cudaStream_t st) {
  return run_frames_any(AdjSrc<float2>{src, tb.status}, B, L, nframes, gu, tb, st);
}

int run_adj_frames_any_f64(const AdjSources<double2>& src, int B, int L, int nframes,
                           double* gu, const Tables& tb, cudaStream_t st) {
  return run_frames_any(AdjSrc<double2>{src, tb.status}, B, L, nframes, gu, tb, st);
}

int run_stft_any_f32x(const StftOp<float, double2, float2>& op, int B, int log2M,
                      const Tables& tb, cudaStream_t st) {
  return run_bluestein<float, float2>(op, B, log2M, tb, st);
}

int run_stft_any_f64(const StftOp<double, double2>& op, int B, int log2M, const Tables& tb,
                     cudaStream_t st) {
  return run_bluestein<double, double2>(op, B, log2M, tb, st);
}

int run_stft_f32(const StftOp<float, float2>& op, int B, int log2L, const Tables& tb,
                 cudaStream_t st) {
  return run_stft<StftOp<float, float2>, float2>(op, B, log2L, tb, st);
}

int run_stft_f64(const StftOp<double, double2>& op, int B, int log2L, const Tables& tb,
                 cudaStream_t st) {
  return run_stft<StftOp<double, double2>, double2>(op, B, log2L, tb, st);
}

int run_stft_f32x(const StftOp<float, double2, float2>& op, int B, int log2L,
                  const Tables& tb, cudaStream_t st) {
  return run_stft<StftOp<float, double2, float2>, double2>(op, B, log2L, tb, st);
}

}  // namespace ssqb
