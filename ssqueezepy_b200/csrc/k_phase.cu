// Phase transforms by differences along time: difftype 'phase' (the
// unwrapped angle of Wx, _ssq_cwt.py:490-496) and difftype 'numeric'
// (phase_cwt_num, _ssq_cwt.py:512-586). Both read one row segment of Wx per
// (signal, scale) and write w of the same width (16 or 8 bytes read and 8 or 4
// written per element); the unwrap is bound by its float64 atan2, one per
// element, the numeric differences by HBM.
#include <cmath>
#include "launch.h"

namespace ssqb {

namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kTwoPiPhase = 6.283185307179586;
constexpr int kPhaseThreads = 512;

// numpy's unwrap correction of one angle difference (period 2 pi, discont
// pi): differences below pi in size are kept; others are moved into
// [-pi, pi) by floor-mod, with -pi taken as +pi when the difference was
// positive. The result is the step of the unwrapped phase.
__device__ __forceinline__ double unwrap_step(double dd) {
  if (fabs(dd) < kPi) return dd;
  double r = fmod(dd + kPi, kTwoPiPhase);
  if (r < 0) r += kTwoPiPhase;
  double m = r - kPi;
  if (m == -kPi && dd > 0) m = kPi;
  return m;
}

template <typename C>
__device__ __forceinline__ double cabs_d(C v) {
  return hypot((double)v.x, (double)v.y);
}

// One CTA per row: w[j] = |step_j| / 2pi for j < M-1, and for the last
// column the size of the whole unwrapped excursion u[M-1] - u[0], the sum of
// the steps (block tree reduction in a fixed order, so deterministic). The
// angles of a tile of columns (plus the next tile's first) are staged in
// shared memory, so each angle is computed once.
template <typename C>
__global__ void __launch_bounds__(kPhaseThreads)
phase_unwrap_kernel(const C* __restrict__ Wx, int ncol, int col0, int M, double gamma,
                    typename RealOf<C>::type* __restrict__ w) {
  typedef typename RealOf<C>::type T;
  __shared__ double part[kPhaseThreads];
  __shared__ double ang[kPhaseThreads + 1];
  const size_t r = blockIdx.x;
  const C* W = Wx + r * (size_t)ncol + col0;
  T* out = w + r * (size_t)M;
  const int tid = threadIdx.x;
  double acc = 0.0;
  for (int j0 = 0; j0 < M - 1; j0 += kPhaseThreads) {
    const int j = j0 + tid;
    C a = W[0];
    if (j < M) {
      a = W[j];
      ang[tid] = atan2((double)a.y, (double)a.x);
    }
    if (tid == 0 && j0 + kPhaseThreads < M) {
      const C b = W[j0 + kPhaseThreads];
      ang[kPhaseThreads] = atan2((double)b.y, (double)b.x);
    }
    __syncthreads();
    if (j < M - 1) {
      const double d = unwrap_step(ang[tid + 1] - ang[tid]);
      acc += d;
      out[j] = cabs_d(a) < gamma ? (T)INFINITY : (T)(fabs(d) / kTwoPiPhase);
    }
    __syncthreads();  // ang is rewritten by the next tile
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double tot = part[0];
    out[M - 1] = cabs_d(W[M - 1]) < gamma ? (T)INFINITY : (T)(fabs(tot) / kTwoPiPhase);
  }
}

template <typename C>
__device__ __forceinline__ C at_wrap(const C* W, int j, int M) {
  j %= M;
  if (j < 0) j += M;
  return W[j];
}

// Periodic differences within the M columns (the reference stacks the last
// two columns before and the first two after the segment):
//   order 1: (W[j+1] - W[j]) / dt, the last column wrapping to W[0]
//   order 2: (-W[j+2] + 4 W[j+1] - 3 W[j]) / (2 dt)
//   order 4: (-W[j+2] + 8 W[j+1] - 8 W[j-1] + W[j-2]) / (12 dt)
// then w = |Im(D / W)| / 2pi, inf where |W| < gamma.
template <typename C>
__global__ void phase_numeric_kernel(const C* __restrict__ Wx, long long rows, int ncol,
                                     int col0, int M, int order, double dt, double gamma,
                                     typename RealOf<C>::type* __restrict__ w) {
  typedef typename RealOf<C>::type T;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * M) return;
  const long long r = i / M;
  const int j = (int)(i % M);
  const C* W = Wx + r * (long long)ncol + col0;
  double dx, dy;
  if (order == 1) {
    const C a = W[j], b = at_wrap(W, j + 1, M);
    dx = ((double)b.x - (double)a.x) / dt;
    dy = ((double)b.y - (double)a.y) / dt;
  } else if (order == 2) {
    const C a = W[j], b = at_wrap(W, j + 1, M), c = at_wrap(W, j + 2, M);
    dx = (-(double)c.x + 4.0 * (double)b.x - 3.0 * (double)a.x) / (2.0 * dt);
    dy = (-(double)c.y + 4.0 * (double)b.y - 3.0 * (double)a.y) / (2.0 * dt);
  } else {
    const C m2 = at_wrap(W, j - 2, M), m1 = at_wrap(W, j - 1, M);
    const C p1 = at_wrap(W, j + 1, M), p2 = at_wrap(W, j + 2, M);
    dx = (-(double)p2.x + 8.0 * (double)p1.x - 8.0 * (double)m1.x + (double)m2.x) / (12.0 * dt);
    dy = (-(double)p2.y + 8.0 * (double)p1.y - 8.0 * (double)m1.y + (double)m2.y) / (12.0 * dt);
  }
  const C a = W[j];
  const double c = (double)a.x, d = (double)a.y;
  const double mag2 = c * c + d * d;
  // Im(D / W) = (dy c - dx d) / |W|^2
  const double v = (dy * c - dx * d) / (mag2 * kTwoPiPhase);
  w[i] = sqrt(mag2) < gamma ? (T)INFINITY : (T)fabs(v);
}

}  // namespace

int run_phase_diff_f32(const float2* Wx, long long rows, int ncol, int col0, int M, int mode,
                       int order, double dt, double gamma, float* w, cudaStream_t st) {
  if (mode == 1) {
    phase_unwrap_kernel<float2><<<(unsigned)rows, kPhaseThreads, 0, st>>>(Wx, ncol, col0, M,
                                                                           gamma, w);
  } else {
    const long long n = rows * M;
    phase_numeric_kernel<float2><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        Wx, rows, ncol, col0, M, order, dt, gamma, w);
  }
  return cudaGetLastError();
}

int run_phase_diff_f64(const double2* Wx, long long rows, int ncol, int col0, int M, int mode,
                       int order, double dt, double gamma, double* w, cudaStream_t st) {
  if (mode == 1) {
    phase_unwrap_kernel<double2><<<(unsigned)rows, kPhaseThreads, 0, st>>>(Wx, ncol, col0, M,
                                                                            gamma, w);
  } else {
    const long long n = rows * M;
    phase_numeric_kernel<double2><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        Wx, rows, ncol, col0, M, order, dt, gamma, w);
  }
  return cudaGetLastError();
}

}  // namespace ssqb
