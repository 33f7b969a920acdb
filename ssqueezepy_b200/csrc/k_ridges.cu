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
#include <cooperative_groups.h>
#include "launch.h"

namespace ssqb {

namespace cg = cooperative_groups;

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

// ---- forward sweep over a thread-block cluster ------------------------------
// CTA c of the cluster owns rows [c R, c R + R) (R = ceil(nf / kRidgeCluster));
// K consecutive lanes share a row, lane k taking the candidates g = k, k+K, ...
// and the K partial minima meet by shuffles. Every CTA holds the whole
// previous column in shared memory, double-buffered: lanes of a row write its
// new value into the other buffer of every CTA through distributed shared
// memory, and one cluster barrier per time step orders the steps. A candidate
// pen[g] + P[f, g] is NaN exactly when pen[g] is (P is finite), so the NaN rule
// of the minimum becomes a per-column flag, set by whoever writes a NaN, in
// three slots: read at step t, written at t + 1, cleared for t + 2. With
// MAXC > 0 the lane's jump penalties P[f, g] (constant in time) sit in
// registers. Global memory stays out of the steps: the barrier's release
// would wait for every outstanding global access, so E for the CTA's rows is
// read into shared memory CHF steps at a time and the accumulated values are
// collected there and written back once per chunk.
constexpr int kRidgeCluster = 8;

template <typename T>
__device__ __forceinline__ T tmin(T a, T b) { return b < a ? b : a; }

template <typename T, int K, int MAXC>
__global__ void __cluster_dims__(kRidgeCluster, 1, 1) __launch_bounds__(1024)
ridge_forward_cluster_kernel(const T* __restrict__ s, T penalty, int nf, int N, int R,
                             int CHF, T* __restrict__ pen) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* prev = reinterpret_cast<T*>(smem_raw);  // [2][nf]
  T* ss = prev + 2 * nf;                      // [nf]
  T* eb = ss + nf;                            // [CHF][R]  E of this chunk's steps
  T* ob = eb + (size_t)CHF * R;               // [CHF][R]  accumulated values
  __shared__ int nanflag[3];
  cg::cluster_group cluster = cg::this_cluster();
  const int c = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int k = tid % K;
  const int fl = tid / K;
  const int f0 = c * R;
  const int f = f0 + fl;
  const int rows = (nf - f0) < R ? (nf - f0 > 0 ? nf - f0 : 0) : R;  // rows owned
  const bool active = fl < rows;
  const unsigned gmask = (K == 32) ? 0xffffffffu
                                   : (((1u << K) - 1u) << ((tid & 31) / K * K));
  int has = 0;
  for (int g = tid; g < nf; g += blockDim.x) {
    const T v = pen[g];
    prev[g] = v;
    ss[g] = s[g];
    has |= (v != v);
  }
  if (tid < 3) nanflag[tid] = 0;
  has = __syncthreads_or(has);
  if (tid == 0) nanflag[0] = has;
  const T sf = active ? ss[f] : (T)0;
  T P[MAXC > 0 ? MAXC : 1];
  if (MAXC > 0) {
#pragma unroll
    for (int i = 0; i < (MAXC > 0 ? MAXC : 1); ++i) {
      const int g = k + i * K;
      P[i] = (active && g < nf) ? jump(penalty, sf, ss[g]) : (T)0;
    }
  }
  cluster.sync();  // every CTA initialised before the first remote write
  // lanes that write other CTAs' buffers: 1..C when a row has more lanes than
  // the cluster has CTAs (lane 0 keeps the chunk store), else all lanes
  const bool remote_lane = (K > kRidgeCluster) ? (k >= 1 && k <= kRidgeCluster) : true;
  for (int t0 = 1; t0 < N; t0 += CHF) {
    const int nst = (N - t0) < CHF ? (N - t0) : CHF;
    // read E[t0 .. t0 + nst) for the owned rows (pen still holds E there)
    for (int q = tid; q < nst * rows; q += blockDim.x) {
      const int tt = q / rows, r = q % rows;
      eb[tt * R + r] = pen[(size_t)(t0 + tt) * nf + f0 + r];
    }
    __syncthreads();
    for (int tt = 0; tt < nst; ++tt) {
      const int t = t0 + tt;
      const T* pv = prev + ((t - 1) & 1) * nf;
      T* pw = prev + (t & 1) * nf;
      const int col_nan = nanflag[(t - 1) % 3];
      if (tid == 0) nanflag[(t + 1) % 3] = 0;
      if (active) {
        T m0 = (T)INFINITY, m1 = (T)INFINITY;
        if (MAXC > 0) {
#pragma unroll
          for (int i = 0; i < (MAXC > 0 ? MAXC : 1); i += 2) {
            const int g0 = k + i * K, g1 = g0 + K;
            if (g0 < nf) m0 = tmin(m0, radd(pv[g0], P[i]));
            if (i + 1 < MAXC && g1 < nf) m1 = tmin(m1, radd(pv[g1], P[i + 1]));
          }
        } else {
          int g = k;
          for (; g + K < nf; g += 2 * K) {
            m0 = tmin(m0, radd(pv[g], jump(penalty, sf, ss[g])));
            m1 = tmin(m1, radd(pv[g + K], jump(penalty, sf, ss[g + K])));
          }
          if (g < nf) m0 = tmin(m0, radd(pv[g], jump(penalty, sf, ss[g])));
        }
        T m = tmin(m0, m1);
#pragma unroll
        for (int o = K / 2; o > 0; o >>= 1) m = tmin(m, __shfl_xor_sync(gmask, m, o));
        if (col_nan) m = (T)NAN;
        const T nv = radd(eb[tt * R + fl], m);
        if (k == 0) ob[tt * R + fl] = nv;
        const bool isnan_v = nv != nv;
        if (K > kRidgeCluster) {
          if (remote_lane) {
            const int r = k - 1;
            *cluster.map_shared_rank(pw + f, r) = nv;
            if (isnan_v) *cluster.map_shared_rank(&nanflag[t % 3], r) = 1;
          }
        } else {
          for (int r = k; r < kRidgeCluster; r += K) {
            *cluster.map_shared_rank(pw + f, r) = nv;
            if (isnan_v) *cluster.map_shared_rank(&nanflag[t % 3], r) = 1;
          }
        }
      }
      cluster.sync();  // every thread of the cluster, every step
    }
    // write the chunk's accumulated values back (ob complete: the last
    // cluster barrier also ordered the CTA's own threads)
    for (int q = tid; q < nst * rows; q += blockDim.x) {
      const int tt = q / rows, r = q % rows;
      pen[(size_t)(t0 + tt) * nf + f0 + r] = ob[tt * R + r];
    }
    __syncthreads();  // eb / ob are rewritten by the next chunk
  }
}

// asynchronous global -> shared copy of one 4- or 8-byte element (cp.async:
// the copy does not pass through registers, so a thread's copies overlap)
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(d), "l"(src) : "memory");
}

// ---- backward sweep: one computing warp, rows staged in shared memory --------
// Warp 0 walks time backwards; lane l holds s[f] for f = l + 32 i in registers
// and reads the rows it needs from a shared-memory chunk of CH time steps
// (pen and E, time-major) that all warps copy in before the chunk starts, the
// next chunk's copy overlapping the walk of the current one.
template <typename T, int I>
__global__ void __launch_bounds__(256)
ridge_backward_staged_kernel(const T* __restrict__ E, const T* __restrict__ pen,
                             const T* __restrict__ s, T penalty, T eps, int nf, int N, int CH,
                             int* __restrict__ ridge) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // two chunk buffers, each [CH + 1][nf] of pen then of E, and [CH] forward argmins
  const size_t rows = (size_t)(CH + 1) * nf;
  T* const base = reinterpret_cast<T*>(smem_raw);
  int* const rbase = reinterpret_cast<int*>(base + 4 * rows);
  // buffer b: pen rows at base + 2 b rows, E rows after them, argmins at rbase + b CH
  const int tid = threadIdx.x, lane = tid & 31;
  // chunk j covers steps t in [hi_j - CH + 1, hi_j], hi_j = N - 2 - j CH, plus
  // row hi_j + 1 (the step above it)
  // copied by threads q0, q0 + 1, ... of the block (all of them before the
  // walk starts, warps 1.. while warp 0 walks)
  auto stage = [&](int j, int b, int q0) {
    const int qt = tid - q0, qs = blockDim.x - q0;
    const int hi = N - 2 - j * CH;
    const int lo = hi - CH + 1 < 0 ? 0 : hi - CH + 1;
    const int n_rows = hi + 1 - lo + 1;  // rows lo .. hi + 1
    const size_t n = (size_t)n_rows * nf;
    const T* gp = pen + (size_t)lo * nf;
    const T* ge = E + (size_t)lo * nf;
    T* sp = base + 2 * (size_t)b * rows;
    T* se = sp + rows;
    int* sr = rbase + b * CH;
    for (size_t q = qt; q < n; q += qs) {
      cp_async_elem(sp + q, gp + q);
      cp_async_elem(se + q, ge + q);
    }
    for (int q = qt; q < hi + 1 - lo; q += qs) cp_async_elem(sr + q, ridge + lo + q);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  T sreg[I];
#pragma unroll
  for (int i = 0; i < I; ++i) {
    const int f = lane + 32 * i;
    sreg[i] = f < nf ? s[f] : (T)0;
  }
  const int nchunks = (N - 1 + CH - 1) / CH;
  int r = ridge[N - 1];
  r = r < 0 ? 0 : (r >= nf ? nf - 1 : r);
  if (nchunks > 0) stage(0, 0, 0);
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  for (int j = 0; j < nchunks; ++j) {
    const int b = j & 1;
    if (tid >= 32) {
      if (j + 1 < nchunks) stage(j + 1, b ^ 1, 32);
      asm volatile("cp.async.wait_all;" ::: "memory");
    } else {
      const int hi = N - 2 - j * CH;
      const int lo = hi - CH + 1 < 0 ? 0 : hi - CH + 1;
      const T* P = base + 2 * (size_t)b * rows;
      const T* Eb = P + rows;
      const int* Rb = rbase + b * CH;
      for (int t = hi; t >= lo; --t) {
        const T* prow = P + (size_t)(t - lo) * nf;         // pen[t, :]
        const size_t o = (size_t)(t + 1 - lo) * nf + r;    // (t + 1, r)
        const T val = rsub(P[o], Eb[o]);
        T sr = (T)0;
#pragma unroll
        for (int i = 0; i < I; ++i)
          if (i == (r >> 5)) sr = sreg[i];
        sr = __shfl_sync(0xffffffffu, sr, r & 31);
        int best = -1;
#pragma unroll
        for (int i = 0; i < I; ++i) {
          const int f = lane + 32 * i;
          if (f < nf) {
            const T d = rsub(val, radd(prow[f], jump(penalty, sr, sreg[i])));
            if (fabs(d) < eps) best = f;
          }
        }
        best = __reduce_max_sync(0xffffffffu, best);
        int rt = best >= 0 ? best : Rb[t - lo];
        if (lane == 0 && best >= 0) ridge[t] = best;
        r = rt < 0 ? 0 : (rt >= nf ? nf - 1 : rt);  // in range by construction
      }
    }
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

constexpr size_t kRidgeFwdSmem = 200 * 1024;

// steps per chunk of the cluster sweep: up to 64, as shared memory allows
template <typename T>
static int fwd_chunk(int nf, int R) {
  const size_t fixed = 3 * (size_t)nf * sizeof(T);
  if (fixed >= kRidgeFwdSmem) return 0;
  const size_t per = 2 * (size_t)R * sizeof(T);
  const size_t c = (kRidgeFwdSmem - fixed) / per;
  return c >= 64 ? 64 : (int)c;
}

template <typename T, int K, int MAXC>
static cudaError_t launch_fwd_cluster(const T* s, T penalty, int nf, int N, T* pen,
                                      cudaStream_t st) {
  const int R = (nf + kRidgeCluster - 1) / kRidgeCluster;
  const int threads = ((R * K + 31) / 32) * 32;
  const int CHF = fwd_chunk<T>(nf, R);
  const size_t smem = (3 * (size_t)nf + 2 * (size_t)CHF * R) * sizeof(T);
  auto k = ridge_forward_cluster_kernel<T, K, MAXC>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  k<<<kRidgeCluster, threads, smem, st>>>(s, penalty, nf, N, R, CHF, pen);
  return cudaGetLastError();
}

// the cluster sweep for up to 1024 rows per CTA with room for a chunk of at
// least 8 steps; otherwise the single-CTA sweep
template <typename T>
static cudaError_t launch_ridge_forward(const T* s, T penalty, int nf, int N, T* pen,
                                        cudaStream_t st) {
  const int R = (nf + kRidgeCluster - 1) / kRidgeCluster;
  if (fwd_chunk<T>(nf, R) >= 8) {
    if (R * 16 <= 1024 && (nf + 15) / 16 <= 32)
      return launch_fwd_cluster<T, 16, 32>(s, penalty, nf, N, pen, st);
    if (R * 8 <= 1024) return launch_fwd_cluster<T, 8, 0>(s, penalty, nf, N, pen, st);
    if (R * 4 <= 1024) return launch_fwd_cluster<T, 4, 0>(s, penalty, nf, N, pen, st);
    if (R <= 1024) return launch_fwd_cluster<T, 1, 0>(s, penalty, nf, N, pen, st);
  }
  const size_t smem = 2 * (size_t)nf * sizeof(T);
  auto fk = ridge_forward_kernel<T>;
  cudaError_t e = cudaFuncSetAttribute(fk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  fk<<<1, 1024, smem, st>>>(s, penalty, nf, N, pen);
  return cudaGetLastError();
}

template <typename T, int I>
static cudaError_t launch_bwd_staged(const T* E, const T* pen, const T* s, T penalty, T eps,
                                     int nf, int N, int CH, size_t smem, int* ridge,
                                     cudaStream_t st) {
  auto k = ridge_backward_staged_kernel<T, I>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  k<<<1, 256, smem, st>>>(E, pen, s, penalty, eps, nf, N, CH, ridge);
  return cudaGetLastError();
}

// staged single-warp walk for nf <= 1024 (32 rows per lane at most) when a
// chunk of at least 4 steps fits; else the block-wide walk
template <typename T>
static cudaError_t launch_ridge_backward(const T* E, const T* pen, const T* s, T penalty, T eps,
                                         int nf, int N, int* ridge, cudaStream_t st) {
  if (N < 2) return cudaSuccess;
  const size_t per_step = 2 * 2 * (size_t)nf * sizeof(T) + 2 * sizeof(int);
  const size_t budget = 160 * 1024;
  int CH = (int)((budget - 2 * 2 * (size_t)nf * sizeof(T)) / per_step);
  if (CH > 64) CH = 64;
  if (nf <= 1024 && CH >= 4) {
    const size_t smem = 2 * 2 * (size_t)(CH + 1) * nf * sizeof(T) + 2 * (size_t)CH * sizeof(int);
    if (nf <= 128) return launch_bwd_staged<T, 4>(E, pen, s, penalty, eps, nf, N, CH, smem, ridge, st);
    if (nf <= 320) return launch_bwd_staged<T, 10>(E, pen, s, penalty, eps, nf, N, CH, smem, ridge, st);
    if (nf <= 512) return launch_bwd_staged<T, 16>(E, pen, s, penalty, eps, nf, N, CH, smem, ridge, st);
    return launch_bwd_staged<T, 32>(E, pen, s, penalty, eps, nf, N, CH, smem, ridge, st);
  }
  ridge_backward_kernel<T><<<1, 1024, 0, st>>>(E, pen, s, penalty, eps, nf, N, ridge);
  return cudaGetLastError();
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
  const unsigned gN = (unsigned)((N + nt - 1) / nt);
  for (int i = 0; i < n_ridges; ++i) {
    ridge_prep_kernel<T><<<gN, nt, 0, st>>>(energy, nf, N, (T)eps, E, pen);
    if ((e = launch_ridge_forward<T>((const T*)s, (T)penalty, nf, N, pen, st))) return e;
    ridge_argmin_kernel<T><<<gN, nt, 0, st>>>(pen, nf, N, ridge);
    if ((e = launch_ridge_backward<T>(E, pen, (const T*)s, (T)penalty, (T)eps, nf, N, ridge,
                                      st)))
      return e;
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
