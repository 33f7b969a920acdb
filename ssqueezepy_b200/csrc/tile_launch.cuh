// Host launchers of the tile kernels, shared by the translation units that
// instantiate them: one pass when L fits a tile, else two passes over row
// tiles sized to the intermediate; batches of signals in chunks.
#pragma once
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
  auto k = tile_pass1<Op, C, LOGL2, SIGN>;
  cudaError_t e = prep(k, smem);
  if (e) return e;
  dim3 grid((1u << log2L) / tile_of<C>(), rows, B);
  k<<<grid, kNT, smem, st>>>(op, tb, Z, log2L, row_lo, rows);
  return cudaGetLastError();
}

template <class Op, typename C, int SIGN, int LOGL1>
static int launch_p2(const Op& op, int B, int log2L, const C* Z, int row_lo, int rows,
                     const Tables& tb, cudaStream_t st) {
  if (int* c = launch_counter()) return ++*c, 0;
  const size_t smem = tile_smem<C>(Op::NARR, LOGL1);
  auto k = tile_pass2<Op, C, LOGL1, SIGN>;
  cudaError_t e = prep(k, smem);
  if (e) return e;
  dim3 grid((1u << log2L) / tile_of<C>(), rows, B);
  k<<<grid, kNT, smem, st>>>(op, tb, Z, log2L, row_lo, rows);
  return cudaGetLastError();
}

template <class Op, typename C, int SIGN>
static int run_single(const Op& op, int B, int nrows, int log2L, const Tables& tb,
                      cudaStream_t st) {
  switch (log2L) {
    case 3: return launch_single<Op, C, SIGN, 3>(op, B, nrows, tb, st);
    case 4: return launch_single<Op, C, SIGN, 4>(op, B, nrows, tb, st);
    case 5: return launch_single<Op, C, SIGN, 5>(op, B, nrows, tb, st);
    case 6: return launch_single<Op, C, SIGN, 6>(op, B, nrows, tb, st);
    case 7: return launch_single<Op, C, SIGN, 7>(op, B, nrows, tb, st);
    case 8: return launch_single<Op, C, SIGN, 8>(op, B, nrows, tb, st);
    case 9: return launch_single<Op, C, SIGN, 9>(op, B, nrows, tb, st);
    case 10: return launch_single<Op, C, SIGN, 10>(op, B, nrows, tb, st);
    case 11: return launch_single<Op, C, SIGN, 11>(op, B, nrows, tb, st);
    case 12:
      if constexpr (tile_of<C>() >= 4096)
        return launch_single<Op, C, SIGN, 12>(op, B, nrows, tb, st);
      else
        return (int)cudaErrorInvalidValue;
    default: return (int)cudaErrorInvalidValue;
  }
}

template <class Op, typename C, int SIGN>
static int run_tile(const Op& op, int B, int nrows, int log2L, C* Z, size_t zcap,
                    const Tables& tb, cudaStream_t st) {
  if (!two_pass<C>(log2L)) return run_single<Op, C, SIGN>(op, B, nrows, log2L, tb, st);
  if (log2L > 22) return (int)cudaErrorInvalidValue;
  const int l2 = log2L / 2, l1 = log2L - l2;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int S = rows_per_tile(zcap, B, Op::NARR, log2L, nrows,
                              (1 << log2L) / tile_of<C>(), 2 * sms);
  for (int r0 = 0; r0 < nrows; r0 += S) {
    const int rows = (nrows - r0) < S ? (nrows - r0) : S;
    int e;
    switch (l2) {
      case 6: e = launch_p1<Op, C, SIGN, 6>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 7: e = launch_p1<Op, C, SIGN, 7>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 8: e = launch_p1<Op, C, SIGN, 8>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 9: e = launch_p1<Op, C, SIGN, 9>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 10: e = launch_p1<Op, C, SIGN, 10>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 11: e = launch_p1<Op, C, SIGN, 11>(op, B, log2L, Z, r0, rows, tb, st); break;
      default: e = (int)cudaErrorInvalidValue;
    }
    if (e) return e;
    switch (l1) {
      case 6: e = launch_p2<Op, C, SIGN, 6>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 7: e = launch_p2<Op, C, SIGN, 7>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 8: e = launch_p2<Op, C, SIGN, 8>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 9: e = launch_p2<Op, C, SIGN, 9>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 10: e = launch_p2<Op, C, SIGN, 10>(op, B, log2L, Z, r0, rows, tb, st); break;
      case 11: e = launch_p2<Op, C, SIGN, 11>(op, B, log2L, Z, r0, rows, tb, st); break;
      default: e = (int)cudaErrorInvalidValue;
    }
    if (e) return e;
  }
  return 0;
}

// Batches: signals go through in chunks whose two-pass intermediate fits
// zcap (at least one signal); each chunk is one run_tile over its signals
// (grid z), the op's descriptor and spectrum pointers advanced to the chunk.
template <class BOp, typename C, int SIGN>
static int run_batch(BOp op, int nsig, int nrows, int log2L, C* Z, size_t zcap,
                     const Tables& tb, cudaStream_t st) {
  int chunk = nsig;
  if (two_pass<C>(log2L)) {
    const size_t per = (size_t)BOp::NARR << log2L;
    const size_t c = zcap / per;
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

}  // namespace ssqb
