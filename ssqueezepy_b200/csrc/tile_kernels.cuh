// Generic tile-FFT kernels: one pass for L <= 4096 (NF sequences per CTA),
// or two passes (four-step) for L = L1*L2 through an intermediate buffer.
//
// For the two-pass form, with input index k = k1 + L1*k2 and output index
// n = L2*n1 + n2 (k1, n1 in [0, L1); k2, n2 in [0, L2)):
//   y[L2*n1 + n2] = sum_k1 w_L1^(k1*n1) * [ w_L^(k1*n2) *
//                   sum_k2 Y[k1 + L1*k2] w_L2^(k2*n2) ]           (w = e^(SIGN 2 pi i / .))
// pass 1: per k1 a length-L2 transform over k2, times w_L^(k1*n2), stored as
//         Z[n2][k1];  pass 2: per n2 a length-L1 transform over k1.
//
// An `Op` supplies the data at both ends:
//   Op::NARR                           arrays transformed together
//   Op::kStoreRowFast                  epilogue iterates rows fastest
//   op.rows()                          number of rows (sequences) per batch item
//   op.load(b, row, k, C out[NARR])    input element k of row `row` of item b
//   op.store(b, row, n, seq, pos, rowbase)
//                                      output element n; its value in array a
//                                      is seq[a][spad(pos)]. In the one-pass
//                                      kernel element m of the same row sits at
//                                      seq[a][spad(rowbase + m)], so ops may
//                                      read partners too (e.g. n and L-n)
#pragma once
#include "fft_tile.cuh"

namespace ssqb {

constexpr int kNT = 256;  // threads per CTA for all tile kernels

template <class Op, typename C, int LOGL, int TILE, int SIGN>
__global__ void __launch_bounds__(kNT)
tile_single(Op op, Tables tb) {
  constexpr int NARR = Op::NARR;
  constexpr int L = 1 << LOGL;
  constexpr int NF = TILE / L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* bufs[NARR];
#pragma unroll
  for (int a = 0; a < NARR; ++a) bufs[a] = base + a * spad_size(TILE);
  C* const(&buf)[NARR] = bufs;
  const int b = blockIdx.z;
  const int row0 = blockIdx.x * NF;
  const int nrows = op.rows();
  int nz = 0;
  for (int e = threadIdx.x; e < TILE; e += kNT) {
    const int f = e >> LOGL, k = e & (L - 1);
    C v[NARR];
    if (row0 + f < nrows) {
      op.load(b, row0 + f, k, v);
    } else {
#pragma unroll
      for (int a = 0; a < NARR; ++a) v[a] = mk((typename RealOf<C>::type)0, (typename RealOf<C>::type)0);
    }
#pragma unroll
    for (int a = 0; a < NARR; ++a) {
      buf[a][spad(e)] = v[a];
      nz |= (v[a].x != 0) | (v[a].y != 0);
    }
  }
  // a tile whose input is all zero transforms to zero: skip the stages
  if (__syncthreads_or(nz)) fft_tile<C, LOGL, NF, kNT, SIGN, NARR>(buf, tw4k<C>(tb));
  for (int e = threadIdx.x; e < TILE; e += kNT) {
    int f, n;
    if (Op::kStoreRowFast) { f = e % NF; n = e / NF; }
    else { f = e >> LOGL; n = e & (L - 1); }
    if (row0 + f < nrows) op.store(b, row0 + f, n, buf, f * L + n, f * L);
  }
}

// pass 1: CTA = (k1 block of NF1 = TILE/L2 columns, row within the row tile,
// batch item). Z layout: [b][row - row_lo][a][n2][k1].
template <class Op, typename C, int LOGL2, int TILE, int SIGN>
__global__ void __launch_bounds__(kNT)
tile_pass1(Op op, Tables tb, C* __restrict__ Z, int log2L, int row_lo, int rows_in_tile) {
  constexpr int NARR = Op::NARR;
  constexpr int L2 = 1 << LOGL2;
  constexpr int NF = TILE / L2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* bufs[NARR];
#pragma unroll
  for (int a = 0; a < NARR; ++a) bufs[a] = base + a * spad_size(TILE);
  C* const(&buf)[NARR] = bufs;
  const int L1 = 1 << (log2L - LOGL2);
  const int b = blockIdx.z;
  const int row = row_lo + blockIdx.y;
  const int k1_0 = blockIdx.x * NF;
  int nz = 0;
  for (int e = threadIdx.x; e < TILE; e += kNT) {
    const int f = e % NF, k2 = e / NF;
    C v[NARR];
    op.load(b, row, k1_0 + f + L1 * k2, v);
#pragma unroll
    for (int a = 0; a < NARR; ++a) {
      buf[a][spad(f * L2 + k2)] = v[a];
      nz |= (v[a].x != 0) | (v[a].y != 0);
    }
  }
  if (__syncthreads_or(nz)) fft_tile<C, LOGL2, NF, kNT, SIGN, NARR>(buf, tw4k<C>(tb));
  const size_t L = size_t(1) << log2L;
  C* zrow = Z + (size_t(b) * rows_in_tile + blockIdx.y) * NARR * L;
  for (int e = threadIdx.x; e < TILE; e += kNT) {
    const int f = e % NF, n2 = e / NF;
    const int k1 = k1_0 + f;
    const uint32_t ex = (uint32_t)(((uint64_t)k1 * (uint64_t)n2) & (L - 1));
    const C w = to_c<C>(unit_root<SIGN>(tb, ex, log2L));
#pragma unroll
    for (int a = 0; a < NARR; ++a)
      zrow[a * L + size_t(n2) * L1 + k1] = cmul(buf[a][spad(f * L2 + n2)], w);
  }
}

// pass 2: CTA = (n2 block of NF2 = TILE/L1 values, row, batch item).
template <class Op, typename C, int LOGL1, int TILE, int SIGN>
__global__ void __launch_bounds__(kNT)
tile_pass2(Op op, Tables tb, const C* __restrict__ Z, int log2L, int row_lo, int rows_in_tile) {
  constexpr int NARR = Op::NARR;
  constexpr int L1 = 1 << LOGL1;
  constexpr int NF = TILE / L1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* bufs[NARR];
#pragma unroll
  for (int a = 0; a < NARR; ++a) bufs[a] = base + a * spad_size(TILE);
  C* const(&buf)[NARR] = bufs;
  const int L2 = 1 << (log2L - LOGL1);
  const int b = blockIdx.z;
  const int row = row_lo + blockIdx.y;
  const int n2_0 = blockIdx.x * NF;
  const size_t L = size_t(1) << log2L;
  const C* zrow = Z + (size_t(b) * rows_in_tile + blockIdx.y) * NARR * L;
  int nz = 0;
  for (int e = threadIdx.x; e < TILE; e += kNT) {
    const int f = e >> LOGL1, k1 = e & (L1 - 1);
#pragma unroll
    for (int a = 0; a < NARR; ++a) {
      const C v = zrow[a * L + size_t(n2_0 + f) * L1 + k1];
      buf[a][spad(e)] = v;
      nz |= (v.x != 0) | (v.y != 0);
    }
  }
  if (__syncthreads_or(nz)) fft_tile<C, LOGL1, NF, kNT, SIGN, NARR>(buf, tw4k<C>(tb));
  for (int e = threadIdx.x; e < TILE; e += kNT) {
    const int f = e % NF, n1 = e / NF;
    op.store(b, row, L2 * n1 + n2_0 + f, buf, f * L1 + n1, f * L1);
  }
}

}  // namespace ssqb
