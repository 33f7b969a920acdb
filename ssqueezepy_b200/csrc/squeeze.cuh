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

// Lane layout: a warp covers G rows x CW = 32/G columns; lane = g*CW + c
// handles column j0 + c of rows i = i0 + g, i0 + G + g, ... The G lanes of a
// column update the shared accumulator in G ordered phases (__syncwarp
// between them), so every bin still receives its rows in ascending order.
// Loads for U row groups are issued before their updates.
template <typename C, class Src, int G, int U>
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
  const size_t base = (size_t)b * na * N + j;
  for (int i0 = 0; i0 < na; i0 += G * U) {
    C v[U];
    typename Src::Pre p[U];
    bool ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * G + g;
      ok[u] = live && i < na;
      if (ok[u]) {
        const size_t o = base + (size_t)i * N;
        v[u] = Wx[o];
        p[u] = src.pre(o);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * G + g;
      int k = -1;
      if (ok[u]) {
        k = src.bin(p[u], v[u], i);
        if (k >= nbins) { set_status(status, DEV_BAD_BIN); k = -1; }
      }
#pragma unroll
      for (int ph = 0; ph < G; ++ph) {
        if (ph == g && k >= 0) {
          C& a = acc[k * CW + c];
          const T w = cs[i];
          a.x += v[u].x * w;
          a.y += v[u].y * w;
        }
        if (G > 1) __syncwarp();
      }
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

// ---- column-tile squeeze from the bin index ---------------------------------
// One warp per tile of 32 consecutive columns of one signal, lane = column.
// The tile's rows stream through shared memory by cp.async (8- or 16-byte
// Wx copies, one per lane and row; the 64-byte index row by four lanes),
// PIPE stages of RS rows in flight, so the copies in flight do not cost
// registers. Rows then accumulate in ascending order into the tile's Tx block
// acc[nbins][32] (lane j touches only column j: two 8-byte accesses per bank
// pair, no conflicts whatever the bins). Q rows at a time: their Q
// accumulator loads are issued together and rows of the group that share a
// bin take the updated value of the previous one from registers, so every
// bin still receives its rows one after the other in ascending order.
// Needs an index pitch that is a multiple of 32 columns and a 16-byte
// aligned index base.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "n"(BYTES)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

#ifndef SSQB_SQ_PIPE
#define SSQB_SQ_PIPE 6
#endif
#ifndef SSQB_SQ_RS
#define SSQB_SQ_RS 16
#endif
#ifndef SSQB_SQ_Q
#define SSQB_SQ_Q 8
#endif
#ifndef SSQB_SQ_RUN
#define SSQB_SQ_RUN 1
#endif
constexpr int kSqPipe = SSQB_SQ_PIPE, kSqRows = SSQB_SQ_RS, kSqQ = SSQB_SQ_Q;

template <typename C>
__host__ __device__ constexpr size_t squeeze_cols_smem(int na, int nbins) {
  return (size_t)nbins * 32 * sizeof(C) + (size_t)kSqPipe * kSqRows * 32 * sizeof(C) +
         (size_t)kSqPipe * kSqRows * 32 * sizeof(uint16_t) +
         (size_t)na * sizeof(typename RealOf<C>::type);
}

template <typename C>
__device__ __forceinline__ void squeeze_cols_body(const C* __restrict__ Wx,
                                                  const uint16_t* __restrict__ idx, int pitch,
                                                  const double* __restrict__ cst, int na,
                                                  int N, int nbins, C* __restrict__ Tx,
                                                  int* status, int tile) {
  typedef typename RealOf<C>::type T;
  constexpr int PIPE = kSqPipe, RS = kSqRows, Q = kSqQ;
  static_assert(RS % Q == 0, "row stage must hold whole row groups");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* acc = reinterpret_cast<C*>(smem_raw);                            // [nbins][32]
  C* sw = acc + (size_t)nbins * 32;                                    // [PIPE][RS][32]
  uint16_t* sk = reinterpret_cast<uint16_t*>(sw + PIPE * RS * 32);     // [PIPE][RS][32]
  T* cs = reinterpret_cast<T*>(sk + PIPE * RS * 32);                  // [na]
  const int lane = threadIdx.x;
  const int j0 = tile * 32;
  const int j = j0 + lane;
  const bool live = j < N;
  const int nst = (na + RS - 1) / RS;
  auto issue = [&](int s) {
    if (s < nst) {
      const int slot = s % PIPE;
#pragma unroll
      for (int r = 0; r < RS; ++r) {
        const int i = s * RS + r;
        if (i < na && live)
          cp_async<sizeof(C)>(sw + (slot * RS + r) * 32 + lane, Wx + (size_t)i * N + j);
      }
#pragma unroll
      for (int q = lane; q < RS * 4; q += 32) {
        const int r = q >> 2, c = q & 3;
        const int i = s * RS + r;
        if (i < na)
          cp_async<16>(sk + (slot * RS + r) * 32 + c * 8, idx + (size_t)i * pitch + j0 + c * 8);
      }
    }
    cp_async_commit();  // empty groups keep the group count uniform
  };
#pragma unroll
  for (int s = 0; s < PIPE - 1; ++s) issue(s);
  {
    float4* a4 = reinterpret_cast<float4*>(acc);
    const int n4 = (int)((size_t)nbins * 32 * sizeof(C) / sizeof(float4));
    for (int e = lane; e < n4; e += 32) a4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = lane; i < na; i += 32) cs[i] = (T)cst[i];
  }
  __syncwarp();
  int curk = -1;  // run-length form: bin of the running sum `cura`
  C cura = mk((T)0, (T)0);
  for (int s = 0; s < nst; ++s) {
    issue(s + PIPE - 1);
    cp_async_wait<PIPE - 1>();
    __syncwarp();
    const int slot = s % PIPE;
    const int rmax = min(RS, na - s * RS);
    const C* wv = sw + slot * RS * 32 + lane;
    const uint16_t* kv = sk + slot * RS * 32 + lane;
#if SSQB_SQ_RUN
    // run-length form: the current bin's sum stays in registers, the
    // accumulator is touched only when a lane's bin changes
    if (live) {
#pragma unroll 4
      for (int r = 0; r < rmax; ++r) {
        const int kk = kv[r * 32];
        if (kk < nbins) {
          if (kk != curk) {
            if (curk >= 0) acc[curk * 32 + lane] = cura;
            cura = acc[kk * 32 + lane];
            curk = kk;
          }
          const C v = wv[r * 32];
          const T w = cs[s * RS + r];
          cura.x += v.x * w;
          cura.y += v.y * w;
        } else if (kk != kNoBin) {
          set_status(status, DEV_BAD_BIN);
        }
      }
    }
#else
#pragma unroll
    for (int r0 = 0; r0 < RS; r0 += Q) {
      if (r0 >= rmax) break;
      int k[Q];
      C v[Q], a[Q];
      T w[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int r = r0 + q;
        k[q] = -1 - q;  // distinct negatives never match another row
        v[q] = wv[r * 32];
        w[q] = cs[s * RS + (r < rmax ? r : 0)];
        if (r < rmax && live) {
          const int kk = kv[r * 32];
          if (kk != kNoBin) {
            if (kk < nbins) k[q] = kk;
            else set_status(status, DEV_BAD_BIN);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) a[q] = k[q] >= 0 ? acc[k[q] * 32 + lane] : mk((T)0, (T)0);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        C b = a[q];
#pragma unroll
        for (int p = 0; p < q; ++p)
          if (k[p] == k[q]) b = a[p];  // the latest earlier row of this bin
        b.x += v[q].x * w[q];
        b.y += v[q].y * w[q];
        a[q] = b;
      }
#pragma unroll
      for (int q = 0; q < Q; ++q)
        if (k[q] >= 0) acc[k[q] * 32 + lane] = a[q];  // in row order: the last one stays
    }
#endif
    __syncwarp();
  }
  if (curk >= 0) acc[curk * 32 + lane] = cura;
  if (live) {
    C* out = Tx + j;
    for (int kk = 0; kk < nbins; ++kk) out[(size_t)kk * N] = acc[kk * 32 + lane];
  }
}

// The same column-tile squeeze with the rows' loads kept in registers, D
// groups of Q rows in flight per lane, and no staging buffers (a smaller
// shared-memory footprint: more warps per SM).
#ifndef SSQB_SQ_REG
#define SSQB_SQ_REG 0
#endif
#ifndef SSQB_SQ_D
#define SSQB_SQ_D 3
#endif
template <typename C>
__host__ __device__ constexpr size_t squeeze_reg_smem(int na, int nbins) {
  return (size_t)nbins * 32 * sizeof(C) + (size_t)na * sizeof(typename RealOf<C>::type);
}

template <typename C>
__device__ __forceinline__ void squeeze_reg_body(const C* __restrict__ Wx,
                                                 const uint16_t* __restrict__ idx, int pitch,
                                                 const double* __restrict__ cst, int na,
                                                 int N, int nbins, C* __restrict__ Tx,
                                                 int* status, int tile) {
  typedef typename RealOf<C>::type T;
  constexpr int Q = kSqQ, D = SSQB_SQ_D;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* acc = reinterpret_cast<C*>(smem_raw);        // [nbins][32]
  T* cs = reinterpret_cast<T*>(acc + (size_t)nbins * 32);
  const int lane = threadIdx.x;
  const int j = tile * 32 + lane;
  const bool live = j < N;
  const int ng = (na + Q - 1) / Q;
  C vb[D][Q];
  int kb[D][Q];
  auto load = [&](int g, C (&v)[Q], int (&k)[Q]) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = g * Q + q;
      k[q] = -1 - q;
      if (g < ng && i < na && live) {
        v[q] = __ldcs(Wx + (size_t)i * N + j);
        k[q] = __ldcs(idx + (size_t)i * pitch + j);
      }
    }
  };
#pragma unroll
  for (int d = 0; d < D; ++d) load(d, vb[d], kb[d]);
  {
    float4* a4 = reinterpret_cast<float4*>(acc);
    const int n4 = (int)((size_t)nbins * 32 * sizeof(C) / sizeof(float4));
    for (int e = lane; e < n4; e += 32) a4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = lane; i < na; i += 32) cs[i] = (T)cst[i];
  }
  __syncwarp();
  int curk = -1;  // run-length form: bin of the running sum `cura`
  C cura = mk((T)0, (T)0);
  for (int g = 0; g < ng; ++g) {
    int k[Q];
    C v[Q], a[Q];
    T w[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      v[q] = vb[0][q];
      int kk = kb[0][q];
      if (kk >= 0) {  // a loaded index: masked, bad or a bin
        if (kk == kNoBin) kk = -1 - q;
        else if (kk >= nbins) { set_status(status, DEV_BAD_BIN); kk = -1 - q; }
      }
      k[q] = kk;
      const int i = g * Q + q;
      w[q] = cs[i < na ? i : 0];
    }
#pragma unroll
    for (int d = 0; d + 1 < D; ++d)
#pragma unroll
      for (int q = 0; q < Q; ++q) { vb[d][q] = vb[d + 1][q]; kb[d][q] = kb[d + 1][q]; }
    load(g + D, vb[D - 1], kb[D - 1]);
#if SSQB_SQ_RUN
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (k[q] >= 0) {
        if (k[q] != curk) {
          if (curk >= 0) acc[curk * 32 + lane] = cura;
          cura = acc[k[q] * 32 + lane];
          curk = k[q];
        }
        cura.x += v[q].x * w[q];
        cura.y += v[q].y * w[q];
      }
    }
#else
#pragma unroll
    for (int q = 0; q < Q; ++q) a[q] = k[q] >= 0 ? acc[k[q] * 32 + lane] : mk((T)0, (T)0);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      C b = a[q];
#pragma unroll
      for (int p = 0; p < q; ++p)
        if (k[p] == k[q]) b = a[p];
      b.x += v[q].x * w[q];
      b.y += v[q].y * w[q];
      a[q] = b;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q)
      if (k[q] >= 0) acc[k[q] * 32 + lane] = a[q];
#endif
  }
  if (curk >= 0) acc[curk * 32 + lane] = cura;
  if (live) {
    C* out = Tx + j;
    for (int kk = 0; kk < nbins; ++kk) __stcs(out + (size_t)kk * N, acc[kk * 32 + lane]);
  }
}

template <typename C>
__host__ __device__ constexpr size_t squeeze_tile_smem(int na, int nbins) {
  return SSQB_SQ_REG ? squeeze_reg_smem<C>(na, nbins) : squeeze_cols_smem<C>(na, nbins);
}
template <typename C>
__device__ __forceinline__ void squeeze_tile_body(const C* Wx, const uint16_t* idx, int pitch,
                                                  const double* cst, int na, int N, int nbins,
                                                  C* Tx, int* status, int tile) {
  if constexpr (SSQB_SQ_REG)
    squeeze_reg_body<C>(Wx, idx, pitch, cst, na, N, nbins, Tx, status, tile);
  else
    squeeze_cols_body<C>(Wx, idx, pitch, cst, na, N, nbins, Tx, status, tile);
}

template <typename C>
__global__ void __launch_bounds__(32)
squeeze_cols_kernel(const C* __restrict__ Wx, const uint16_t* __restrict__ idx, int pitch,
                    const double* __restrict__ cst, int na, int N, int nbins,
                    C* __restrict__ Tx, int* status) {
  const size_t b = blockIdx.y;
  squeeze_tile_body<C>(Wx + b * na * N, idx + b * na * pitch, pitch, cst, na, N, nbins,
                       Tx + b * nbins * N, status, blockIdx.x);
}

// Batches of uneven lengths: signal blockIdx.y per its descriptor; column
// tiles past its length return at once.
template <typename C>
__global__ void __launch_bounds__(32)
squeeze_cols_batch_kernel(const C* __restrict__ Wx, const uint16_t* __restrict__ idx,
                          const SigDesc* __restrict__ desc, C* __restrict__ Tx, int* status) {
  const SigDesc& d = desc[blockIdx.y];
  if ((int)blockIdx.x * 32 >= d.N) return;
  squeeze_tile_body<C>(Wx + d.out_off, idx + d.idx_off, d.idx_pitch, d.weights, d.na, d.N,
                       d.nbins, Tx + d.out_off, status, blockIdx.x);
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
  squeeze_body<C, IdxSrc<C>, G, U>(Wx + d.out_off, src, d.weights, d.na, d.N, d.nbins,
                                   Tx + d.out_off, status, 0, blockIdx.x);
}

}  // namespace ssqb
