// Deterministic synchrosqueeze: Tx[k(i,j), j] += Wx[i,j] * c_i.
//
// One warp owns 32 consecutive time columns of one signal and keeps their
// whole Tx column block, nbins x 32, in shared memory. Lane l walks the rows
// i = 0..na-1 of column j0+l in ascending order, the order of the reference's
// per-column loop (algos.py:879-895), so every bin accumulates in a fixed
// order: no atomics, results independent of scheduling. Loads of Wx and of
// the bin source are issued U rows ahead of the shared-memory updates.
#pragma once
#include "ssqb_ops.cuh"

namespace ssqb {

// bin from a precomputed uint16 index (kNoBin = masked)
template <typename C>
struct IdxSrc {
  const uint16_t* idx;
  int pitch, N;  // idx rows of `pitch` columns; Wx rows of N
  struct Pre { uint16_t k; };
  __device__ __forceinline__ Pre pre(size_t o) const {
    return Pre{__ldg(idx + (o / N) * pitch + o % N)};
  }
  __device__ __forceinline__ int bin(const Pre& p, C, int) const {
    return p.k == kNoBin ? -1 : (int)p.k;
  }
};

// bin from (Wx, dWx) on the fly: ssqueeze_fast (algos.py:126-150)
template <typename C>
struct PhaseSrc {
  const C* dWx;
  const double* sfs;   // null for the CWT
  BinDev bins;
  double gamma;
  int* status;
  struct Pre { C d; };
  __device__ __forceinline__ Pre pre(size_t o) const { return Pre{dWx[o]}; }
  __device__ __forceinline__ int bin(const Pre& p, C v, int i) const {
    const uint16_t k = phase_bin(v, p.d, sfs ? sfs[i] : 0.0, sfs != nullptr, bins,
                                 gamma, status, nullptr);
    return k == kNoBin ? -1 : (int)k;
  }
};

// bin from a precomputed phase transform w (inf = masked): indexed_sum_onfly
// (algos.py:153-250)
template <typename C>
struct WSrc {
  typedef typename RealOf<C>::type T;
  const T* w;
  BinDev bins;
  int* status;
  struct Pre { T w; };
  __device__ __forceinline__ Pre pre(size_t o) const { return Pre{w[o]}; }
  __device__ __forceinline__ int bin(const Pre& p, C, int) const {
    if (isinf(p.w)) return -1;
    const int k = bin_of(bins, (double)p.w);
    if (k < 0 || k >= bins.nbins) { set_status(status, DEV_BAD_BIN); return -1; }
    return k;
  }
};

constexpr int kSqU = 8;  // rows in flight per lane

template <typename C, class Src>
__global__ void __launch_bounds__(32)
squeeze_kernel(const C* __restrict__ Wx, Src src, const double* __restrict__ cst,
               int na, int N, int nbins, C* __restrict__ Tx, int* status) {
  typedef typename RealOf<C>::type T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* acc = reinterpret_cast<C*>(smem_raw);           // [nbins][32]
  T* cs = reinterpret_cast<T*>(acc + (size_t)nbins * 32);  // [na]
  const int lane = threadIdx.x;
  const int b = blockIdx.y;
  const int j = blockIdx.x * 32 + lane;
  const bool live = j < N;
  for (int k = lane; k < nbins * 32; k += 32) acc[k] = mk((T)0, (T)0);
  for (int i = lane; i < na; i += 32) cs[i] = (T)cst[i];
  __syncwarp();
  const size_t base = (size_t)b * na * N + j;
  int i = 0;
  for (; i + kSqU <= na; i += kSqU) {
    C v[kSqU];
    typename Src::Pre p[kSqU];
#pragma unroll
    for (int u = 0; u < kSqU; ++u) {
      const size_t o = base + (size_t)(i + u) * N;
      if (live) { v[u] = Wx[o]; p[u] = src.pre(o); }
    }
#pragma unroll
    for (int u = 0; u < kSqU; ++u) {
      if (!live) continue;
      const int k = src.bin(p[u], v[u], i + u);
      if (k >= nbins) { set_status(status, DEV_BAD_BIN); continue; }
      if (k >= 0) {
        C& a = acc[k * 32 + lane];
        const T c = cs[i + u];
        a.x += v[u].x * c;
        a.y += v[u].y * c;
      }
    }
  }
  for (; i < na; ++i) {
    if (!live) break;
    const size_t o = base + (size_t)i * N;
    const C v = Wx[o];
    const typename Src::Pre p = src.pre(o);
    const int k = src.bin(p, v, i);
    if (k >= nbins) { set_status(status, DEV_BAD_BIN); continue; }
    if (k >= 0) {
      C& a = acc[k * 32 + lane];
      const T c = cs[i];
      a.x += v.x * c;
      a.y += v.y * c;
    }
  }
  __syncwarp();
  if (live) {
    C* out = Tx + (size_t)b * nbins * N + j;
    for (int k = 0; k < nbins; ++k) out[(size_t)k * N] = acc[k * 32 + lane];
  }
}

}  // namespace ssqb
