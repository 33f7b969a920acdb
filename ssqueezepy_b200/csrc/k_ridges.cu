// Time-frequency ridge extraction (ridge_extraction.py:11-232, the serial
// code path): forward-backward tracking of the minimum accumulated
//   E[f, t] = -log(energy[f, t] / max_f energy[:, t] + eps)
// plus the jump penalty P[f, f'] = penalty * (s_f - s_f')^2, in the
// arithmetic type of the input (float32 for complex64).
//
// The forward sweep is sequential in time and parallel in frequency: one
// CTA keeps the previous column in shared memory and forms, for every f,
// min_f' (pen[f', t-1] + P[f, f']) (NaN propagates, as numpy's amin). The
// backward sweep re-walks time from the end; at each step the last f whose
// accumulated value matches within eps replaces the forward argmin. Sums are
// rounded separately (no fused multiply-add) so they equal the reference's.
#include "launch.h"

namespace ssqb {

template <typename T> __device__ __forceinline__ T radd(T a, T b);
template <> __device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
template <typename T> __device__ __forceinline__ T rsub(T a, T b);
template <> __device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
template <> __device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
template <typename T> __device__ __forceinline__ T rmul(T a, T b);
template <> __device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }

// penalty * (a - b)^2, rounded as numpy's penalty * subtract.outer(s, s)**2
template <typename T>
__device__ __forceinline__ T jump(T penalty, T a, T b) {
  const T d = rsub(a, b);
  return rmul(penalty, rmul(d, d));
}

// energy = |Tf|^2 (np.abs(Tf)**2)
template <typename C>
__global__ void ridge_energy_kernel(const C* __restrict__ Tf, size_t n,
                                    typename RealOf<C>::type* __restrict__ energy) {
  typedef typename RealOf<C>::type T;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const C z = Tf[i];
  // |z| rounded once to T (float: through double, as a correctly rounded hypot)
  const T a = (T)hypot((double)z.x, (double)z.y);
  energy[i] = rmul(a, a);
}

// per column t: E[t, f] = -log(energy[f, t] / max_f energy + eps), pen = E.
// E and pen are time-major (t, f): the sweeps read one time step contiguous.
template <typename T>
__global__ void ridge_prep_kernel(const T* __restrict__ energy, int nf, int N, T eps,
                                  T* __restrict__ E, T* __restrict__ pen) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N) return;
  T mx = energy[t];
  bool nan = mx != mx;
  for (int f = 1; f < nf; ++f) {
    const T v = energy[(size_t)f * N + t];
    if (v != v) nan = true;
    if (v > mx) mx = v;
  }
  if (nan) mx = (T)NAN;
  for (int f = 0; f < nf; ++f) {
    const T e = -log(radd(energy[(size_t)f * N + t] / mx, eps));
    E[(size_t)t * nf + f] = e;
    pen[(size_t)t * nf + f] = e;
  }
}

// forward sweep, one CTA: pen[f, t] = E[f, t] + min_f' (pen[f', t-1] + P[f, f'])
template <typename T>
__global__ void __launch_bounds__(1024)
ridge_forward_kernel(const T* __restrict__ s, T penalty, int nf, int N, T* __restrict__ pen) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* prev = reinterpret_cast<T*>(smem_raw);   // [nf]
  T* ss = prev + nf;                          // [nf]
  for (int f = threadIdx.x; f < nf; f += blockDim.x) {
    prev[f] = pen[f];
    ss[f] = s[f];
  }
  __syncthreads();
  for (int t = 1; t < N; ++t) {
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
      const T sf = ss[f];
      T m = radd(prev[0], jump(penalty, sf, ss[0]));
      bool nan = m != m;
      for (int g = 1; g < nf; ++g) {
        const T v = radd(prev[g], jump(penalty, sf, ss[g]));
        nan |= v != v;
        m = v < m ? v : m;
      }
      if (nan) m = (T)NAN;
      const size_t o = (size_t)t * nf + f;
      pen[o] = radd(pen[o], m);
    }
    __syncthreads();
    for (int f = threadIdx.x; f < nf; f += blockDim.x) prev[f] = pen[(size_t)t * nf + f];
    __syncthreads();
  }
}

// per column: first index of the minimum over f (the first NaN if any)
template <typename T>
__global__ void ridge_argmin_kernel(const T* __restrict__ pen, int nf, int N,
                                    int* __restrict__ ridge) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N) return;
  int best = 0;
  const T* row = pen + (size_t)t * nf;
  T m = row[0];
  if (m == m) {
    for (int f = 1; f < nf; ++f) {
      const T v = row[f];
      if (v != v) { best = f; break; }
      if (v < m) { m = v; best = f; }
    }
  }
  ridge[t] = best;
}

// backward sweep, one CTA: the last f with |val - (pen[f, t] + P[r, f])| < eps
template <typename T>
__global__ void __launch_bounds__(1024)
ridge_backward_kernel(const T* __restrict__ E, const T* __restrict__ pen,
                      const T* __restrict__ s, T penalty, T eps, int nf, int N,
                      int* __restrict__ ridge) {
  __shared__ int warp_best[32];
  __shared__ int r_next;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) r_next = ridge[N - 1];
  __syncthreads();
  for (int t = N - 2; t >= 0; --t) {
    const int r = r_next;
    const size_t o = (size_t)(t + 1) * nf + r;
    const T val = rsub(pen[o], E[o]);
    const T sr = s[r];
    int best = -1;
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
      const T d = rsub(val, radd(pen[(size_t)t * nf + f], jump(penalty, sr, s[f])));
      if (fabs(d) < eps) best = f;  // f ascends per thread: the last one wins
    }
    for (int k = 16; k > 0; k >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, k));
    if (lane == 0) warp_best[wid] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
      int b = -1;
      for (int w = 0; w < nw; ++w) b = max(b, warp_best[w]);
      if (b >= 0) ridge[t] = b;
      r_next = ridge[t];
    }
    __syncthreads();
  }
}

// ridge parameters and removal of the extracted ridge's band from energy:
// rows [ridx - bw, ridx + bw) with Python slice semantics (a negative start
// counts from the end)
template <typename T>
__global__ void ridge_finish_kernel(const int* __restrict__ ridge, const T* __restrict__ scales,
                                    int nf, int N, int bw, int col, int ncol,
                                    T* __restrict__ energy, int* __restrict__ idx_out,
                                    T* __restrict__ f_out, T* __restrict__ e_out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N) return;
  const int r = ridge[t];
  idx_out[(size_t)t * ncol + col] = r;
  if (f_out) f_out[(size_t)t * ncol + col] = scales[r];
  if (e_out) e_out[(size_t)t * ncol + col] = energy[(size_t)r * N + t];
  long long a = (long long)r - bw, b = (long long)r + bw;
  if (a < 0) a += nf;
  if (b < 0) b += nf;
  a = a < 0 ? 0 : (a > nf ? nf : a);
  b = b < 0 ? 0 : (b > nf ? nf : b);
  for (long long f = a; f < b; ++f) energy[(size_t)f * N + t] = (T)0;
}

template <typename C>
static int run_ridges_t(const C* Tf, int nf, int N, const void* s, const void* scales,
                        double penalty, int n_ridges, int bw, double eps, int* idx_out,
                        void* f_out, void* e_out, void* ws, cudaStream_t st) {
  typedef typename RealOf<C>::type T;
  const size_t n = (size_t)nf * N;
  T* energy = (T*)ws;
  T* E = energy + n;
  T* pen = E + n;
  int* ridge = (int*)(pen + n);
  const int nt = 256;
  ridge_energy_kernel<C><<<(unsigned)((n + nt - 1) / nt), nt, 0, st>>>(Tf, n, energy);
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  const size_t smem = 2 * (size_t)nf * sizeof(T);
  auto fk = ridge_forward_kernel<T>;
  if ((e = cudaFuncSetAttribute(fk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
    return e;
  const unsigned gN = (unsigned)((N + nt - 1) / nt);
  for (int i = 0; i < n_ridges; ++i) {
    ridge_prep_kernel<T><<<gN, nt, 0, st>>>(energy, nf, N, (T)eps, E, pen);
    fk<<<1, 1024, smem, st>>>((const T*)s, (T)penalty, nf, N, pen);
    ridge_argmin_kernel<T><<<gN, nt, 0, st>>>(pen, nf, N, ridge);
    ridge_backward_kernel<T><<<1, 1024, 0, st>>>(E, pen, (const T*)s, (T)penalty, (T)eps, nf,
                                                 N, ridge);
    ridge_finish_kernel<T><<<gN, nt, 0, st>>>(ridge, (const T*)scales, nf, N, bw, i, n_ridges,
                                              energy, idx_out, (T*)f_out, (T*)e_out);
    if ((e = cudaGetLastError())) return e;
  }
  return 0;
}

size_t ridges_workspace(int nf, int N, bool f64) {
  return 3 * (size_t)nf * N * (f64 ? sizeof(double) : sizeof(float)) + (size_t)N * sizeof(int);
}

int run_ridges(const void* Tf, int nf, int N, const void* s, const void* scales, double penalty,
               int n_ridges, int bw, double eps, bool f64, int* idx_out, void* f_out,
               void* e_out, void* ws, cudaStream_t st) {
  if (f64)
    return run_ridges_t<double2>((const double2*)Tf, nf, N, s, scales, penalty, n_ridges, bw,
                                 eps, idx_out, f_out, e_out, ws, st);
  return run_ridges_t<float2>((const float2*)Tf, nf, N, s, scales, penalty, n_ridges, bw, eps,
                              idx_out, f_out, e_out, ws, st);
}

}  // namespace ssqb
