// Deterministic synchrosqueeze: Tx[k(i,j), j] += Wx[i,j] * c_i.
//
// One warp owns a few consecutive time columns of one signal and keeps their
// whole Tx column block, nbins x columns, in shared memory. Each bin of a
// column receives its rows in ascending order, the order of the reference's
// per-column loop (algos.py:879-895): no atomics, results independent of
// scheduling.
#pragma once
#include "ssqb_ops.cuh"

namespace ssqb {

// Sources give the bin of entry (row, j) of Wx, at flat offset o = row * N + j
// (row counts over all signals' rows): pre() issues its loads, bin() decodes.

// bin from a precomputed uint16 index (kNoBin = masked)
template <typename C>
struct IdxSrc {
  const uint16_t* idx;
  int pitch, N;  // idx rows of `pitch` columns; Wx rows of N
  struct Pre { uint16_t k; };
  __device__ __forceinline__ Pre pre(size_t, size_t row, int j) const {
    return Pre{__ldg(idx + row * pitch + j)};
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
  __device__ __forceinline__ Pre pre(size_t o, size_t, int) const { return Pre{dWx[o]}; }
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
  __device__ __forceinline__ Pre pre(size_t o, size_t, int) const { return Pre{w[o]}; }
  __device__ __forceinline__ int bin(const Pre& p, C, int) const {
    if (isinf(p.w)) return -1;
    const int k = bin_of(bins, (double)p.w);
    if (k < 0 || k >= bins.nbins) { set_status(status, DEV_BAD_BIN); return -1; }
    return k;
  }
};

// Lane layout: a warp covers G rows x CW = 32/G columns; lane = g*CW + c
// handles column j0 + c of rows i = i0 + g, i0 + G + g, ... The G lanes of a
// column update the shared accumulator in G ordered phases (__syncwarp
// between them), so every bin still receives its rows in ascending order.
// Loads for U row groups are issued before their updates; with PIPE the
// next U row groups' loads are also in flight during those updates.
template <typename C, class Src, int G, int U, bool PIPE = false>
__device__ __forceinline__ void squeeze_body(const C* __restrict__ Wx, const Src& src,
                                             const double* __restrict__ cst, int na, int N,
                                             int nbins, C* __restrict__ Tx, int* status,
                                             int b, int tile) {
  typedef typename RealOf<C>::type T;
  constexpr int CW = 32 / G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* acc = reinterpret_cast<C*>(smem_raw);                   // [nbins][CW]
  T* cs = reinterpret_cast<T*>(acc + (size_t)nbins * CW);   // [na]
  const int lane = threadIdx.x;
  const int g = lane / CW, c = lane % CW;
  const int j = tile * CW + c;
  const bool live = j < N;
  for (int k = lane; k < nbins * CW; k += 32) acc[k] = mk((T)0, (T)0);
  for (int i = lane; i < na; i += 32) cs[i] = (T)cst[i];
  __syncwarp();
  const size_t row0 = (size_t)b * na;
  const size_t base = row0 * N + j;
  struct Batch {
    C v[U];
    typename Src::Pre p[U];
    bool ok[U];
  };
  // loads of rows i0 + u*G + g, u < U
  auto load = [&](Batch& bt, int i0) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * G + g;
      bt.ok[u] = live && i < na;
      if (bt.ok[u]) {
        const size_t o = base + (size_t)i * N;
        bt.v[u] = Wx[o];
        bt.p[u] = src.pre(o, row0 + i, j);
      }
    }
  };
  // their updates, in ascending row order per bin
  auto update = [&](const Batch& bt, int i0) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * G + g;
      int k = -1;
      if (bt.ok[u]) {
        k = src.bin(bt.p[u], bt.v[u], i);
        if (k >= nbins) { set_status(status, DEV_BAD_BIN); k = -1; }
      }
#pragma unroll
      for (int ph = 0; ph < G; ++ph) {
        if (ph == g && k >= 0) {
          C& a = acc[k * CW + c];
          const T w = cs[i];
          a.x += bt.v[u].x * w;
          a.y += bt.v[u].y * w;
        }
        if (G > 1) __syncwarp();
      }
    }
  };
  constexpr int STEP = G * U;
  if constexpr (PIPE) {
    // two batches in flight: the next batch's loads are issued before this
    // batch's updates
    Batch A, B;
    load(A, 0);
    for (int i0 = 0; i0 < na; i0 += 2 * STEP) {
      if (i0 + STEP < na) load(B, i0 + STEP);
      update(A, i0);
      if (i0 + STEP >= na) break;
      if (i0 + 2 * STEP < na) load(A, i0 + 2 * STEP);
      update(B, i0 + STEP);
    }
  } else {
    for (int i0 = 0; i0 < na; i0 += STEP) {
      Batch bt;
      load(bt, i0);
      update(bt, i0);
    }
  }
  __syncwarp();
  C* out = Tx + (size_t)b * nbins * N + tile * CW;
  const int ncol = min(CW, N - tile * CW);
  for (int e = lane; e < nbins * CW; e += 32) {
    const int k = e / CW, cc = e % CW;
    if (cc < ncol) out[(size_t)k * N + cc] = acc[e];
  }
}

template <typename C, class Src, int G, int U>
__global__ void __launch_bounds__(32)
squeeze_kernel(const C* __restrict__ Wx, Src src, const double* __restrict__ cst,
               int na, int N, int nbins, C* __restrict__ Tx, int* status) {
  squeeze_body<C, Src, G, U>(Wx, src, cst, na, N, nbins, Tx, status, blockIdx.y, blockIdx.x);
}

// Batches of uneven lengths: signal blockIdx.y per its descriptor; column
// tiles past its length return at once.
template <typename C, int G, int U>
__global__ void __launch_bounds__(32)
squeeze_batch_kernel(const C* __restrict__ Wx, const uint16_t* __restrict__ idx,
                     const SigDesc* __restrict__ desc, C* __restrict__ Tx, int* status) {
  const SigDesc& d = desc[blockIdx.y];
  if ((int)blockIdx.x * (32 / G) >= d.N) return;
  IdxSrc<C> src{idx + d.idx_off, d.idx_pitch, d.N};
  squeeze_body<C, IdxSrc<C>, G, U, true>(Wx + d.out_off, src, d.weights, d.na, d.N, d.nbins,
                                   Tx + d.out_off, status, 0, blockIdx.x);
}

}  // namespace ssqb
