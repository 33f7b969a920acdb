// Squeeze kernel instantiations and launchers.
#include "launch.h"
#include "squeeze.cuh"

namespace ssqb {

// Lane layout G (rows per warp instruction): the accumulator of a warp is
// nbins x 32/G; G = 4 keeps it small enough for about ten warps per SM.
// U: row groups whose loads are issued together. Measured, one signal at
// N = 160,000 / 60,000 (293 / 277 rows): U = 8 0.373 / 0.139 ms, 4: 0.562 /
// 0.213, 12: 0.48 / 0.18, 16: 0.436 / 0.172. The batch kernel (per-signal
// descriptors) over 256 signals of 4,096-65,536 samples, whose Wx comes
// mostly from DRAM: U = 16 25.5 ms, 8: 38.6, 12: 40.1; with the next 16 row
// groups' loads in flight during the updates (PIPE) 22.2 ms. The one-signal
// kernel with PIPE: 0.379 ms (U = 8) / 0.371 (U = 4) against 0.373.
#ifndef SSQB_SQ_G
#define SSQB_SQ_G 4
#endif
#ifndef SSQB_SQ_U
#define SSQB_SQ_U 8
#endif
#ifndef SSQB_SQB_U
#define SSQB_SQB_U 16
#endif

template <typename C, class Src>
static int launch_sq(const C* Wx, const Src& src, const double* cst, int B, int na, int N,
                     int nbins, C* Tx, int* status, cudaStream_t st) {
  typedef typename RealOf<C>::type T;
  constexpr int G = SSQB_SQ_G, U = SSQB_SQ_U, CW = 32 / G;
  const size_t smem = (size_t)nbins * CW * sizeof(C) + (size_t)na * sizeof(T);
  auto k = squeeze_kernel<C, Src, G, U>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  dim3 grid((N + CW - 1) / CW, B);
  k<<<grid, 32, smem, st>>>(Wx, src, cst, na, N, nbins, Tx, status);
  return cudaGetLastError();
}

template <typename C>
static int run_sq(const C* Wx, int src_kind, const void* src, int idx_pitch,
                  const double* sfs, const BinDev& bins, double gamma, const double* cst,
                  int B, int na, int N, int nbins, C* Tx, int* status, cudaStream_t st) {
  typedef typename RealOf<C>::type T;
  switch (src_kind) {
    case 0: {
      IdxSrc<C> s{(const uint16_t*)src, idx_pitch, N};
      return launch_sq(Wx, s, cst, B, na, N, nbins, Tx, status, st);
    }
    case 1: {
      PhaseSrc<C> s{(const C*)src, sfs, bins, gamma, status};
      return launch_sq(Wx, s, cst, B, na, N, nbins, Tx, status, st);
    }
    case 2: {
      WSrc<C> s{(const T*)src, bins, status};
      return launch_sq(Wx, s, cst, B, na, N, nbins, Tx, status, st);
    }
    default:
      return (int)cudaErrorInvalidValue;
  }
}

int run_squeeze_batch_f32(const float2* Wx, const uint16_t* idx, const SigDesc* desc,
                          int nsig, int max_na, int max_N, float2* Tx, int* status,
                          cudaStream_t st) {
  if (int* c = launch_counter()) return ++*c, 0;
  constexpr int G = SSQB_SQ_G, U = SSQB_SQB_U, CW = 32 / G;
  const size_t smem = (size_t)max_na * CW * sizeof(float2) + (size_t)max_na * sizeof(float);
  auto k = squeeze_batch_kernel<float2, G, U>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  dim3 grid((max_N + CW - 1) / CW, nsig);
  k<<<grid, 32, smem, st>>>(Wx, idx, desc, Tx, status);
  return cudaGetLastError();
}

int run_squeeze_f32(const float2* Wx, int src_kind, const void* src, int idx_pitch,
                    const double* sfs, const BinDev& bins, double gamma, const double* cst,
                    int B, int na, int N, int nbins, float2* Tx, int* status,
                    cudaStream_t st) {
  return run_sq<float2>(Wx, src_kind, src, idx_pitch, sfs, bins, gamma, cst, B, na, N,
                        nbins, Tx, status, st);
}

int run_squeeze_f64(const double2* Wx, int src_kind, const void* src, int idx_pitch,
                    const double* sfs, const BinDev& bins, double gamma, const double* cst,
                    int B, int na, int N, int nbins, double2* Tx, int* status,
                    cudaStream_t st) {
  return run_sq<double2>(Wx, src_kind, src, idx_pitch, sfs, bins, gamma, cst, B, na, N,
                         nbins, Tx, status, st);
}

}  // namespace ssqb

namespace ssqb {

// x[b, j] = sum_i Re Wx[b, i, j] * w_i + x_mean[b] * mw; one thread per
// column, rows in ascending order (float64 accumulation).
template <typename C>
__global__ void icwt_kernel(const C* __restrict__ Wx, const double* __restrict__ w,
                            const double* __restrict__ x_mean, double mw, int na, int N,
                            typename RealOf<C>::type* __restrict__ x) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (j >= N) return;
  const C* p = Wx + (size_t)b * na * N + j;
  double acc = 0.0;
  int i = 0;
  for (; i + 4 <= na; i += 4) {
    const double r0 = (double)p[(size_t)(i + 0) * N].x, r1 = (double)p[(size_t)(i + 1) * N].x;
    const double r2 = (double)p[(size_t)(i + 2) * N].x, r3 = (double)p[(size_t)(i + 3) * N].x;
    acc += r0 * w[i];
    acc += r1 * w[i + 1];
    acc += r2 * w[i + 2];
    acc += r3 * w[i + 3];
  }
  for (; i < na; ++i) acc += (double)p[(size_t)i * N].x * w[i];
  if (x_mean) acc += x_mean[b] * mw;
  x[(size_t)b * N + j] = (typename RealOf<C>::type)acc;
}

int run_icwt(const void* Wx, const double* w, const double* x_mean, double mean_weight,
             int B, int na, int N, int precision, void* x, cudaStream_t st) {
  dim3 grid((N + 255) / 256, B);
  if (precision == 0)
    icwt_kernel<float2><<<grid, 256, 0, st>>>((const float2*)Wx, w, x_mean, mean_weight, na,
                                              N, (float*)x);
  else
    icwt_kernel<double2><<<grid, 256, 0, st>>>((const double2*)Wx, w, x_mean, mean_weight,
                                               na, N, (double*)x);
  return cudaGetLastError();
}

// Inverse synchrosqueeze (_ssq_cwt.py:366-400): for column j, component n
// sums Re Tx[k, j] over rows k in [lo, hi] with hi = clip(cc + cw, 0, nrows),
// lo = clip(cc - cw, 0, nrows) (an empty range where cc = -1); the last
// output row sums the rows outside every component's range. K = 0: the sum
// of all rows. Rows ascending, float64 accumulation, times `scale`.
constexpr int kMaxIssqComponents = 16;

template <typename C>
__global__ void issq_kernel(const C* __restrict__ Tx, int nrows, int N,
                            const int* __restrict__ cc, const int* __restrict__ cw, int K,
                            double scale, void* __restrict__ xv) {
  typedef typename RealOf<C>::type T;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  int lo[kMaxIssqComponents], hi[kMaxIssqComponents];
  double part[kMaxIssqComponents];
  for (int n = 0; n < K; ++n) {
    const long long c = cc[(size_t)j * K + n], w = cw[(size_t)j * K + n];
    long long up = c + w, dn = c - w;
    up = up < 0 ? 0 : (up > nrows ? nrows : up);
    dn = dn < 0 ? 0 : (dn > nrows ? nrows : dn);
    if (c == -1) { up = 0; dn = 1; }
    lo[n] = (int)dn;
    hi[n] = (int)up;
    part[n] = 0.0;
  }
  double rest = 0.0;
  for (int k = 0; k < nrows; ++k) {
    const double v = (double)Tx[(size_t)k * N + j].x;
    bool in = false;
    for (int n = 0; n < K; ++n) {
      if (k >= lo[n] && k <= hi[n]) {
        part[n] += v;
        in = true;
      }
    }
    if (!in) rest += v;
  }
  if (K > 0) {  // components: float64 rows, as the reference's np.zeros((K + 1, N))
    double* x = (double*)xv;
    for (int n = 0; n < K; ++n) x[(size_t)n * N + j] = part[n] * scale;
    x[(size_t)K * N + j] = rest * scale;
  } else {
    ((T*)xv)[j] = (T)(rest * scale);
  }
}

int run_issq(const void* Tx, int nrows, int N, const int* cc, const int* cw, int K,
             double scale, int precision, void* x, cudaStream_t st) {
  const dim3 grid((N + 255) / 256);
  if (precision == 0)
    issq_kernel<float2><<<grid, 256, 0, st>>>((const float2*)Tx, nrows, N, cc, cw, K, scale,
                                              x);
  else
    issq_kernel<double2><<<grid, 256, 0, st>>>((const double2*)Tx, nrows, N, cc, cw, K, scale,
                                               x);
  return cudaGetLastError();
}

}  // namespace ssqb
