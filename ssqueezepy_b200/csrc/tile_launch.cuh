// Host launchers of the tile kernels, shared by the translation units that
// instantiate them: one pass when L fits a tile, else two passes over row
// tiles sized to the intermediate; batches of signals in chunks.
#pragma once
#include <type_traits>
#include "launch.h"

namespace ssqb {

static inline int ilog2(int n) { int m = 0; while ((1 << m) < n) ++m; return m; }

template <class K>
static cudaError_t prep(K kernel, size_t smem) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem);
}

template <class Op, typename C, int SIGN, int LOGL>
static int launch_single(const Op& op, int B, int nrows, const Tables& tb, cudaStream_t st) {
  if (int* c = launch_counter()) return ++*c, 0;
  constexpr int NF = tile_of<C>() / (1 << LOGL);
  const size_t smem = tile_smem<C>(Op::NARR, LOGL);
  auto k = tile_single<Op, C, LOGL, SIGN>;
  cudaError_t e = prep(k, smem);
  if (e) return e;
  dim3 grid((nrows + NF - 1) / NF, 1, B);
  k<<<grid, kNT, smem, st>>>(op, tb);
  return cudaGetLastError();
}

template <class Op, typename C, int SIGN, int LOGL2>
static int launch_p1(const Op& op, int B, int log2L, C* Z, int row_lo, int rows,
                     const Tables& tb, cudaStream_t st) {
  if (int* c = launch_counter()) return ++*c, 0;
  const size_t smem = tile_smem<C>(Op::NARR, LOGL2);
  dim3 grid((1u << log2L) / tile_of<C>(), rows, B);
  auto k = tile_pass1<Op, C, LOGL2, SIGN>;
  cudaError_t e = prep(k, smem);
  if (e) return e;
  k<<<grid, kNT, smem, st>>>(op, tb, Z, log2L, row_lo, rows);
  return cudaGetLastError();
}

template <class Op, typename C, int SIGN, int LOGL1>
static int launch_p2(const Op& op, int B, int log2L, const C* Z, int row_lo, int rows,
                     const Tables& tb, cudaStream_t st) {
  if (int* c = launch_counter()) return ++*c, 0;
  const size_t smem = tile_smem<C>(Op::NARR, LOGL1);
  dim3 grid((1u << log2L) / tile_of<C>(), rows, B);
  auto k = tile_pass2<Op, C, LOGL1, SIGN>;
  cudaError_t e = prep(k, smem);
  if (e) return e;
  k<<<grid, kNT, smem, st>>>(op, tb, Z, log2L, row_lo, rows);
  return cudaGetLastError();
}

// v in [LO, HI] -> f(std::integral_constant<int, v>), compile-time bounded
template <int LO, int HI, class F>
static int dispatch_log(int v, const F& f) {
  if constexpr (LO > HI) {
    return (int)cudaErrorInvalidValue;
  } else {
    if (v == LO) return f(std::integral_constant<int, LO>{});
    return dispatch_log<LO + 1, HI>(v, f);
  }
}

template <typename C> constexpr int tile_log() {
  int m = 0;
  while ((1 << m) < tile_of<C>()) ++m;
  return m;
}

template <class Op, typename C, int SIGN>
static int run_single(const Op& op, int B, int nrows, int log2L, const Tables& tb,
                      cudaStream_t st) {
  return dispatch_log<3, tile_log<C>()>(log2L, [&](auto k) {
    return launch_single<Op, C, SIGN, decltype(k)::value>(op, B, nrows, tb, st);
  });
}

template <class Op, typename C, int SIGN>
static int run_rows(const Op& op, int B, int log2L, C* Z, int r0, int rows, const Tables& tb,
                    cudaStream_t st) {
  const int l2 = log2L / 2, l1 = log2L - l2;
  int e = dispatch_log<3, tile_log<C>()>(l2, [&](auto k) {
    return launch_p1<Op, C, SIGN, decltype(k)::value>(op, B, log2L, Z, r0, rows, tb, st);
  });
  if (e) return e;
  return dispatch_log<3, tile_log<C>()>(l1, [&](auto k) {
    return launch_p2<Op, C, SIGN, decltype(k)::value>(op, B, log2L, Z, r0, rows, tb, st);
  });
}

template <class Op, typename C, int SIGN>
static int run_tile(const Op& op, int B, int nrows, int log2L, C* Z, size_t zcap,
                    const Tables& tb, cudaStream_t st) {
  if (!two_pass<C>(log2L)) return run_single<Op, C, SIGN>(op, B, nrows, log2L, tb, st);
  if (log2L > 22) return (int)cudaErrorInvalidValue;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
  }
  const int cpr = (1 << log2L) / tile_of<C>();
  // two half-size intermediates when the rows need more than one tile of each
  const size_t per = (size_t)B * Op::NARR << log2L;
  bool dual = SSQB_DUAL_STREAM && zcap / 2 >= per && (size_t)nrows * per > zcap / 2;
  const bool dry = launch_counter() != nullptr;
  AuxStream* ax = (dual && !dry) ? aux_stream() : nullptr;
  if (dual && !dry && !ax) dual = false;
  const size_t cap = dual ? zcap / 2 : zcap;
  const int S = rows_per_tile(cap, B, Op::NARR, log2L, nrows, cpr, 2 * sms);
  if (!dual || dry) {
    int t = 0;
    for (int r0 = 0; r0 < nrows; r0 += S, ++t) {
      const int e = run_rows<Op, C, SIGN>(op, B, log2L, Z + (dual ? (t & 1) * cap : 0), r0,
                                          (nrows - r0) < S ? (nrows - r0) : S, tb, st);
      if (e) return e;
    }
    return 0;
  }
  cudaError_t ce = cudaEventRecord(ax->fork, st);
  if (!ce) ce = cudaStreamWaitEvent(ax->s, ax->fork, 0);
  if (ce) return ce;
  int e = 0;
  int t = 0;
  for (int r0 = 0; r0 < nrows && !e; r0 += S, ++t) {
    const int rows = (nrows - r0) < S ? (nrows - r0) : S;
    e = run_rows<Op, C, SIGN>(op, B, log2L, Z + (t & 1) * cap, r0, rows, tb,
                              (t & 1) ? ax->s : st);
  }
  // join even after a failed launch, so the caller's stream never runs ahead
  ce = cudaEventRecord(ax->join, ax->s);
  if (!ce) ce = cudaStreamWaitEvent(st, ax->join, 0);
  return e ? e : (int)ce;
}

// Batches: signals go through in chunks whose two-pass intermediate fits
// zcap (at least one signal); each chunk is one run_tile over its signals
// (grid z), the op's descriptor and spectrum pointers advanced to the chunk.
template <class BOp, typename C, int SIGN>
static int run_batch(BOp op, int nsig, int nrows, int log2L, C* Z, size_t zcap,
                     const Tables& tb, cudaStream_t st) {
  int chunk = nsig;
  if (two_pass<C>(log2L)) {
    // chunks of signals whose row fits half the intermediate, so that row
    // tiles can alternate between two streams
    const size_t per = (size_t)BOp::NARR << log2L;
    const size_t c = (SSQB_DUAL_STREAM ? zcap / 2 : zcap) / per;
    chunk = c < 1 ? 1 : (c > (size_t)nsig ? nsig : (int)c);
  }
  const size_t Npad = (size_t)1 << log2L;
  for (int s0 = 0; s0 < nsig; s0 += chunk) {
    BOp o = op;
    o.desc += s0;
    o.xh += (size_t)s0 * Npad;
    const int n = (nsig - s0) < chunk ? (nsig - s0) : chunk;
    const int e = run_tile<BOp, C, SIGN>(o, n, nrows, log2L, Z, zcap, tb, st);
    if (e) return e;
  }
  return 0;
}

// Band-limited single pass over rows [r0, r0 + nrows) whose bands fit M =
// 2^logM bins: per chunk of signals (their band inputs Zb fit the
// intermediate), band_prep then band_single.
template <class Op, typename C, int SIGN, int LOGM>
static int launch_band(const Op& op, int B, int log2L, C* Z, int r0, int nrows,
                       const Tables& tb, cudaStream_t st) {
  if (int* c = launch_counter()) return *c += 2, 0;
  constexpr int NF = tile_of<C>() / (1 << LOGM);
  band_prep<Op, C><<<dim3(nrows, 1, B), kNT, 0, st>>>(op, Z, r0, nrows, LOGM);
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  const size_t smem = tile_smem<C>(Op::NARR, LOGM);
  dim3 grid((1u << (log2L - LOGM)) / NF, nrows, B);
  auto k = band_single<Op, C, LOGM, SIGN>;
  e = prep(k, smem);
  if (e) return e;
  k<<<grid, kNT, smem, st>>>(op, tb, Z, log2L, r0, nrows);
  return cudaGetLastError();
}

template <typename C> constexpr int band_max_log() { return tile_log<C>() - 1; }

template <class Op, typename C, int SIGN>
static int run_band(const Op& op, int B, int log2L, int logM, C* Z, size_t zcap, int r0,
                    int nrows, const Tables& tb, cudaStream_t st) {
  const size_t per = (size_t)Op::NARR << logM;  // one signal-row of band inputs
  const size_t rc = zcap / per;                  // signal-rows that fit
  if (rc < 1) return (int)cudaErrorInvalidValue;
  int nb = 1, rstep = nrows;
  if ((size_t)nrows <= rc) {
    const size_t q = rc / nrows;
    nb = q < (size_t)B ? (int)q : B;
  } else {
    rstep = (int)rc;
  }
  for (int b0 = 0; b0 < B; b0 += nb) {
    const int n = B - b0 < nb ? B - b0 : nb;
    for (int q0 = 0; q0 < nrows; q0 += rstep) {
      const int nr = nrows - q0 < rstep ? nrows - q0 : rstep;
      const int e = dispatch_log<3, band_max_log<C>()>(logM, [&](auto k) {
        return launch_band<Op, C, SIGN, decltype(k)::value>(op.shifted(b0), n, log2L, Z,
                                                            r0 + q0, nr, tb, st);
      });
      if (e) return e;
    }
  }
  return 0;
}

// Signals of one call in chunks when all of them need more than half of the
// intermediate per row: each chunk's row fits half of the L2 budget, so its
// row tiles alternate between two streams (ops with `shifted(b0)`).
#ifndef SSQB_CHUNK_SIGNALS
#define SSQB_CHUNK_SIGNALS 1
#endif
template <class Op, typename C, int SIGN>
static int run_tile_signals(const Op& op, int B, int nrows, int log2L, C* Z, size_t zcap,
                            const Tables& tb, cudaStream_t st) {
  const size_t per_sig = (size_t)Op::NARR << log2L;
  if (!SSQB_CHUNK_SIGNALS || !SSQB_DUAL_STREAM || B < 2 || !two_pass<C>(log2L) ||
      (size_t)B * per_sig <= zcap / 2)
    return run_tile<Op, C, SIGN>(op, B, nrows, log2L, Z, zcap, tb, st);
  const size_t budget = cwt_z_budget(log2L) / sizeof(C);
  const size_t half = budget / 2;
  size_t bc = half / per_sig;
  if (bc < 1) bc = 1;
  const int Bc = (int)bc;
  size_t cap = 2 * bc * per_sig;
  if (cap < budget) cap = budget;
  if (cap > zcap) cap = zcap;
  for (int b0 = 0; b0 < B; b0 += Bc) {
    const int n = (B - b0) < Bc ? (B - b0) : Bc;
    const int e = run_tile<Op, C, SIGN>(op.shifted(b0), n, nrows, log2L, Z, cap, tb, st);
    if (e) return e;
  }
  return 0;
}

}  // namespace ssqb
