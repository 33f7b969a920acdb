// Tile-FFT kernels: one pass for L <= TILE (NF rows per CTA), or two passes
// (four-step) for L = L1*L2 through an intermediate buffer Z.
//
// For the two-pass form, with input index k = k1 + L1*k2 and output index
// n = L2*n1 + n2 (k1, n1 in [0, L1); k2, n2 in [0, L2)):
//   y[L2*n1 + n2] = sum_k1 w_L1^(k1*n1) * [ w_L^(k1*n2) *
//                   sum_k2 Y[k1 + L1*k2] w_L2^(k2*n2) ]        (w = e^(SIGN 2 pi i / .))
// pass 1: per k1 a length-L2 transform over k2, times w_L^(k1*n2), stored as
//         Z[n2][k1];  pass 2: per n2 a length-L1 transform over k1.
//
// An `Op` supplies the data at both ends:
//   Op::NARR                             arrays transformed together
//   Op::kDirect                          true: outputs go straight to op.store
//   op.rows()                            rows (sequences) per batch item
//   op.load(b, row, k, C (&v)[NARR])     input element k of row `row`
//   op.store(b, row, n, C (&v)[NARR])    output element n (kDirect)
//   op.store_smem<LY>(b, row, n, buf, f) output element n read from shared
//                                        memory row f (!kDirect; may read
//                                        partner elements, e.g. L-n)
#pragma once
#include "fft_tile.cuh"

namespace ssqb {

constexpr int kNT = 256;  // threads per CTA for all tile kernels

template <typename C> __host__ __device__ constexpr int tile_of() {
  return FftCfg<C>::TILE;
}

// CTAs per SM requested from the compiler (register budget per thread)
#ifndef SSQB_FP64_MINBLOCKS
#define SSQB_FP64_MINBLOCKS 2
#endif
template <typename C> struct MinBlocks { static constexpr int v = 2; };
template <> struct MinBlocks<double2> { static constexpr int v = SSQB_FP64_MINBLOCKS; };

// An op with `kRolledStore` has its outputs stored in a rolled loop: one
// copy of a long store (e.g. a wavelet evaluation) instead of R.
template <class T, class = void> struct RolledStore : std::false_type {};
template <class T>
struct RolledStore<T, std::void_t<decltype(T::kRolledStore)>>
    : std::bool_constant<T::kRolledStore> {};

// Storer handing each output to op.store. Single pass: row = row0 + f,
// index m; pass 2: row fixed, index L2*m + n2_0 + f (mul = L2, add = n2_0).
template <class Op, typename C>
struct StoreEach {
  static constexpr int NARR = Op::NARR;
  const Op& op;
  int b, row0, nrows, mul, add;
  template <int R>
  __device__ __forceinline__ void item(int f, int m0, int stride, C (&a)[R], C (&z)[R]) const {
    const bool single = (nrows != 0x7fffffff);
    const int row = single ? row0 + f : row0;
    if (single && row >= nrows) return;
    auto one = [&](int r) {
      C v[NARR];
      v[0] = a[r];
      v[NARR - 1] = z[r];
      const int m = m0 + r * stride;
      op.store(b, row, single ? m : mul * m + add + f, v);
    };
    if constexpr (RolledStore<Op>::value) {
#pragma unroll 1
      for (int r = 0; r < R; ++r) one(r);
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) one(r);
    }
  }
};

// Pass-1 storer: Z[a][n2][k1] = v * w_L^(k1*n2) for n2 = m0 + r*stride, the
// twiddles by recurrence from two table values (float64).
template <typename C, int NARR, int SIGN>
struct Pass1Store {
  const Tables& tb;
  C* zrow;
  int k1_0, L1, log2L;
  template <int R>
  __device__ __forceinline__ void item(int f, int m0, int stride, C (&a)[R], C (&z)[R]) const {
    const int k1 = k1_0 + f;
    const uint64_t mask = ((uint64_t)1 << log2L) - 1;
    const size_t L = (size_t)1 << log2L;
    double2 w = unit_root<SIGN>(tb, (uint32_t)(((uint64_t)k1 * (uint64_t)m0) & mask), log2L);
    const double2 s =
        unit_root<SIGN>(tb, (uint32_t)(((uint64_t)k1 * (uint64_t)stride) & mask), log2L);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const C wc = to_c<C>(w);
      const size_t o = size_t(m0 + r * stride) * L1 + k1;
      zrow[o] = cmul(a[r], wc);
      if constexpr (NARR > 1) zrow[L + o] = cmul(z[r], wc);
      w = mk(w.x * s.x - w.y * s.y, w.x * s.y + w.y * s.x);
    }
  }
};

// Mapping of the first stage of tile_single: MAP_J unless the op asks for
// rows-fastest loads (kMapIn = MAP_F, e.g. inputs stored frame-minor).
template <class T, class = void> struct MapIn { static constexpr int value = MAP_J; };
template <class T>
struct MapIn<T, std::void_t<decltype(T::kMapIn)>> { static constexpr int value = T::kMapIn; };

// Pass-1 loader: input k1_0 + f + L1*m of row `row`. Ops with a split load
// get a gather that issues the R spectrum loads of an item (only those in
// the row's wavelet band) before any wavelet arithmetic.
template <class BOp, typename C, int NARR, class = void>
struct P1Loader {
  const BOp& op;
  int b, row, k1_0, L1;
  __device__ __forceinline__ void operator()(int f, int m, C (&v)[NARR]) const {
    op.load(b, row, k1_0 + f + L1 * m, v);
  }
};
template <class BOp, typename C, int NARR>
struct P1Loader<BOp, C, NARR, std::enable_if_t<BOp::kSplitLoad>> {
  static constexpr bool kGather = true;
  const BOp& op;
  int b, row, k1_0, L1, klo, khi;
  __device__ __forceinline__ void operator()(int f, int m, C (&v)[NARR]) const {
    op.load(b, row, k1_0 + f + L1 * m, v);
  }
  template <int R>
  __device__ __forceinline__ void gather(int f, int j, int stride, C (&t)[R][NARR]) const {
    double2 raw[R];
#pragma unroll
    for (int r = 0; r < R; ++r) raw[r] = op.raw(b, k1_0 + f + L1 * (j + r * stride), klo, khi);
    if constexpr (std::is_same<C, float2>::value) {
      // float32 transforms: one copy of the wavelet code (rolled loop) keeps
      // the kernel small enough for the instruction cache (measured faster;
      // with float64 transforms the unrolled form is faster)
      double ps[R];
#pragma unroll 1
      for (int r = 0; r < R; ++r) {
        const int k = k1_0 + f + L1 * (j + r * stride);
        const int kk = (k <= (op.Npad >> 1)) ? k : k - op.Npad;
        ps[r] = (kk >= klo && kk <= khi) ? op.psi(row, k) : 0.0;
      }
#pragma unroll
      for (int r = 0; r < R; ++r)
        op.apply(k1_0 + f + L1 * (j + r * stride), raw[r], ps[r], t[r]);
    } else {
      // float64 transforms: all R evaluations inlined (loops unrolled 2 and 4
      // measured 0.1 % and 1.5 % slower at N = 160,000; the wavelet's formula
      // branch hoisted out of the R evaluations, 2-4 % slower)
#pragma unroll
      for (int r = 0; r < R; ++r)
        op.finish(b, row, k1_0 + f + L1 * (j + r * stride), raw[r], t[r]);
    }
  }
};

template <class BOp, typename C, int NARR>
__device__ __forceinline__ P1Loader<BOp, C, NARR> make_p1_loader(const BOp& op, int b, int row,
                                                                  int k1_0, int L1) {
  if constexpr (HasGather<P1Loader<BOp, C, NARR>>::value) {
    int klo, khi;
    op.band_bins(row, klo, khi);
    return P1Loader<BOp, C, NARR>{op, b, row, k1_0, L1, klo, khi};
  } else {
    return P1Loader<BOp, C, NARR>{op, b, row, k1_0, L1};
  }
}

template <class Op, typename C, int LOGL, int SIGN>
__global__ void __launch_bounds__(kNT, MinBlocks<C>::v)
tile_single(Op op, Tables tb) {
  constexpr int NARR = Op::NARR;
  constexpr int TILE = tile_of<C>();
  constexpr int L = 1 << LOGL;
  constexpr int NF = TILE / L;
  typedef Layout<C, LOGL, NF> LY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* bufs[NARR];
#pragma unroll
  for (int a = 0; a < NARR; ++a) bufs[a] = base + a * LY::ARR;
  C* const(&buf)[NARR] = bufs;
  const auto bop = op.bind(blockIdx.z);  // per-signal op (batches of uneven lengths)
  const int b = Op::kBatch ? 0 : blockIdx.z;
  const int row0 = blockIdx.x * NF;
  const int nrows = bop.rows();
  if (row0 >= nrows) return;
  auto ld = [&](int f, int m, C (&v)[NARR]) {
    if (row0 + f < nrows) {
      bop.load(b, row0 + f, m, v);
    } else {
#pragma unroll
      for (int a = 0; a < NARR; ++a)
        v[a] = mk((typename RealOf<C>::type)0, (typename RealOf<C>::type)0);
    }
  };
  typedef decltype(op.bind(0)) BOp;
  constexpr int MI = MapIn<BOp>::value;
  if constexpr (Op::kDirect) {
    StoreEach<BOp, C> st{bop, b, row0, nrows, 1, 0};
    fft_rows<C, LOGL, NF, kNT, SIGN, NARR, MI, MAP_J, true>(buf, seg_table<C>(tb), ld, st);
  } else {
    StoreEach<BOp, C> st{bop, b, row0, nrows, 1, 0};
    fft_rows<C, LOGL, NF, kNT, SIGN, NARR, MI, MAP_J, false>(buf, seg_table<C>(tb), ld, st);
    for (int e = threadIdx.x; e < TILE; e += kNT) {
      const int f = e % NF, n = e / NF;  // rows fastest: coalesced (row, n) outputs
      if (row0 + f < nrows) bop.template store_smem<LY>(b, row0 + f, n, buf, f);
    }
  }
}

// pass 1: CTA = (k1 block of NF = TILE/L2 columns, row within the row tile,
// batch item). Z layout: [b][row - row_lo][a][n2][k1].
template <class Op, typename C, int LOGL2, int SIGN>
__global__ void __launch_bounds__(kNT, MinBlocks<C>::v)
tile_pass1(Op op, Tables tb, C* __restrict__ Z, int log2L, int row_lo, int rows_in_tile) {
  constexpr int NARR = Op::NARR;
  constexpr int TILE = tile_of<C>();
  constexpr int L2 = 1 << LOGL2;
  constexpr int NF = TILE / L2;
  typedef Layout<C, LOGL2, NF> LY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* bufs[NARR];
#pragma unroll
  for (int a = 0; a < NARR; ++a) bufs[a] = base + a * LY::ARR;
  C* const(&buf)[NARR] = bufs;
  const int L1 = 1 << (log2L - LOGL2);
  const auto bop = op.bind(blockIdx.z);
  const int b = Op::kBatch ? 0 : blockIdx.z;
  const int row = row_lo + blockIdx.y;
  if (row >= bop.rows()) return;  // signals with fewer rows (uneven batches)
  const int k1_0 = blockIdx.x * NF;
  const size_t L = size_t(1) << log2L;
  C* zrow = Z + (size_t(blockIdx.z) * rows_in_tile + blockIdx.y) * NARR * L;
  typedef decltype(op.bind(0)) BOp;
  const auto ld = make_p1_loader<BOp, C, NARR>(bop, b, row, k1_0, L1);
  if constexpr (HasGather<P1Loader<BOp, C, NARR>>::value) {
    // A band narrower than L1 bins leaves whole columns k1 without inputs
    // (column k1 holds the bins k = k1 mod L1). If none of this CTA's
    // columns meets the band, its transforms are exactly zero.
    const int W = ld.khi - ld.klo + 1;
    if (W < L1) {
      const int r0 = ((ld.klo % L1) + L1) % L1;
      bool any = false;
#pragma unroll
      for (int f = 0; f < NF; ++f) any |= ((k1_0 + f - r0 + L1) % L1) < W;
      if (!any) {
        const C zero = mk((typename RealOf<C>::type)0, (typename RealOf<C>::type)0);
        for (int e = threadIdx.x; e < NF * L2; e += kNT) {
          const size_t o = (size_t)(e / NF) * L1 + k1_0 + (e % NF);
#pragma unroll
          for (int a = 0; a < NARR; ++a) zrow[a * L + o] = zero;
        }
        return;
      }
    }
  }
  Pass1Store<C, NARR, SIGN> st{tb, zrow, k1_0, L1, log2L};
  fft_rows<C, LOGL2, NF, kNT, SIGN, NARR, MAP_F, MAP_F, true>(buf, seg_table<C>(tb), ld, st);
}

// pass 2: CTA = (n2 block of NF = TILE/L1 values, row, batch item).
template <class Op, typename C, int LOGL1, int SIGN>
__global__ void __launch_bounds__(kNT, MinBlocks<C>::v)
tile_pass2(Op op, Tables tb, const C* __restrict__ Z, int log2L, int row_lo,
           int rows_in_tile) {
  constexpr int NARR = Op::NARR;
  constexpr int TILE = tile_of<C>();
  constexpr int L1 = 1 << LOGL1;
  constexpr int NF = TILE / L1;
  typedef Layout<C, LOGL1, NF> LY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* bufs[NARR];
#pragma unroll
  for (int a = 0; a < NARR; ++a) bufs[a] = base + a * LY::ARR;
  C* const(&buf)[NARR] = bufs;
  const int L2 = 1 << (log2L - LOGL1);
  const auto bop = op.bind(blockIdx.z);
  const int b = Op::kBatch ? 0 : blockIdx.z;
  const int row = row_lo + blockIdx.y;
  if (row >= bop.rows()) return;
  const int n2_0 = blockIdx.x * NF;
  const size_t L = size_t(1) << log2L;
  const C* zrow = Z + (size_t(blockIdx.z) * rows_in_tile + blockIdx.y) * NARR * L;
  auto ld = [&](int f, int m, C (&v)[NARR]) {
#pragma unroll
    for (int a = 0; a < NARR; ++a) v[a] = zrow[a * L + size_t(n2_0 + f) * L1 + m];
  };
  typedef decltype(op.bind(0)) BOp;
  StoreEach<BOp, C> st{bop, b, row, 0x7fffffff, L2, n2_0};
  fft_rows<C, LOGL1, NF, kNT, SIGN, NARR, MAP_J, MAP_F, true>(buf, seg_table<C>(tb), ld, st);
}

// ---- band-limited single pass ---------------------------------------------------
// A row whose wavelet band (signed bins [klo, khi], op.band_bins) fits in M
// bins needs no four-step. With D = L / M and n = D a + n2 (n2 < D, a < M),
//   y[D a + n2] = e^{SIGN 2 pi i klo n / L}
//                 sum_{m<M} (Zb[m] e^{SIGN 2 pi i m n2 / L}) e^{SIGN 2 pi i m a / M},
// Zb[m] = the transform's input at bin klo + m (zero past khi): D transforms of
// length M of the twiddled band. A CTA takes NF = TILE / M consecutive
// residues n2, so each output index a gives NF consecutive columns.
//
// band_prep: Zb[(b, r)][a][m] for rows row0 + r (both arrays), the band's
// inputs formed once per row (spectrum x wavelet in float64, as pass 1).
template <class Op, typename C>
__global__ void __launch_bounds__(kNT)
band_prep(Op op, C* __restrict__ Zb, int row0, int nrows, int logM) {
  constexpr int NARR = Op::NARR;
  const auto bop = op.bind(blockIdx.z);
  const int b = Op::kBatch ? 0 : blockIdx.z;
  const int row = row0 + blockIdx.x;
  if (row >= bop.na) return;  // signals with fewer rows (uneven batches)
  const int M = 1 << logM;
  int klo, khi;
  bop.band_bins(row, klo, khi);
  C* zb = Zb + ((size_t)blockIdx.z * nrows + blockIdx.x) * NARR * M;
  if (khi - klo + 1 > M && threadIdx.x == 0) set_status(bop.status, DEV_BAD_INDEX);
  for (int m = threadIdx.x; m < M; m += kNT) {
    const int kk = klo + m;
    C v[NARR];
    if (kk <= khi) {
      const int k = kk < 0 ? kk + bop.Npad : kk;
      bop.apply(k, bop.raw(b, k, klo, khi), bop.psi(row, k), v);
    } else {
#pragma unroll
      for (int a = 0; a < NARR; ++a)
        v[a] = mk((typename RealOf<C>::type)0, (typename RealOf<C>::type)0);
    }
#pragma unroll
    for (int a = 0; a < NARR; ++a) zb[a * M + m] = v[a];
  }
}

// first-stage gather of the twiddled band: inputs j + r*stride of residue
// n2_0 + f, twiddles by recurrence from two table values
template <typename C, int NARR, int SIGN>
struct BandLoader {
  static constexpr bool kGather = true;
  const Tables& tb;
  const C* zb;
  int M, n2_0, log2L;
  __device__ __forceinline__ void operator()(int f, int m, C (&v)[NARR]) const {
    const uint64_t mask = ((uint64_t)1 << log2L) - 1;
    const C w = to_c<C>(unit_root<SIGN>(tb, (uint32_t)(((uint64_t)m * (n2_0 + f)) & mask),
                                        log2L));
#pragma unroll
    for (int a = 0; a < NARR; ++a) v[a] = cmul(__ldg(zb + a * M + m), w);
  }
  template <int R>
  __device__ __forceinline__ void gather(int f, int j, int stride, C (&t)[R][NARR]) const {
    const uint64_t mask = ((uint64_t)1 << log2L) - 1;
    const uint64_t n2 = (uint64_t)(n2_0 + f);
    C raw[R][NARR];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int a = 0; a < NARR; ++a) raw[r][a] = __ldg(zb + a * M + j + r * stride);
    double2 w = unit_root<SIGN>(tb, (uint32_t)(((uint64_t)j * n2) & mask), log2L);
    const double2 s = unit_root<SIGN>(tb, (uint32_t)(((uint64_t)stride * n2) & mask), log2L);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const C wc = to_c<C>(w);
#pragma unroll
      for (int a = 0; a < NARR; ++a) t[r][a] = cmul(raw[r][a], wc);
      w = mk(w.x * s.x - w.y * s.y, w.x * s.y + w.y * s.x);
    }
  }
};

// storer: output a = m0 + r*stride of residue n2_0 + f is column
// n = D a + n2_0 + f, times e^{SIGN 2 pi i klo n / L}, handed to op.store
template <class BOp, typename C, int SIGN>
struct BandStore {
  static constexpr int NARR = BOp::NARR;
  const BOp& op;
  const Tables& tb;
  int b, row, D, n2_0, klo, log2L;
  template <int R>
  __device__ __forceinline__ void item(int f, int m0, int stride, C (&a)[R], C (&z)[R]) const {
    const int64_t L = (int64_t)1 << log2L;
    const int n0 = D * m0 + n2_0 + f;      // column of r = 0
    const int64_t kl = ((int64_t)klo % L + L) % L;
    double2 p = unit_root<SIGN>(tb, (uint32_t)((kl * n0) & (L - 1)), log2L);
    const double2 s = unit_root<SIGN>(tb, (uint32_t)((kl * D * stride) & (L - 1)), log2L);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const C pc = to_c<C>(p);
      C v[NARR];
      v[0] = cmul(a[r], pc);
      v[NARR - 1] = cmul(z[r], pc);
      op.store(b, row, n0 + D * stride * r, v);
      p = mk(p.x * s.x - p.y * s.y, p.x * s.y + p.y * s.x);
    }
  }
};

// CTA = (NF residues, row row0 + blockIdx.y, batch item)
template <class Op, typename C, int LOGM, int SIGN>
__global__ void __launch_bounds__(kNT, MinBlocks<C>::v)
band_single(Op op, Tables tb, const C* __restrict__ Zb, int log2L, int row0, int nrows) {
  constexpr int NARR = Op::NARR;
  constexpr int TILE = tile_of<C>();
  constexpr int M = 1 << LOGM;
  constexpr int NF = TILE / M;
  typedef Layout<C, LOGM, NF> LY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* base = reinterpret_cast<C*>(smem_raw);
  C* bufs[NARR];
#pragma unroll
  for (int a = 0; a < NARR; ++a) bufs[a] = base + a * LY::ARR;
  C* const(&buf)[NARR] = bufs;
  const auto bop = op.bind(blockIdx.z);
  const int b = Op::kBatch ? 0 : blockIdx.z;
  const int row = row0 + blockIdx.y;
  if (row >= bop.na) return;
  int klo, khi;
  bop.band_bins(row, klo, khi);
  const C* zb = Zb + ((size_t)blockIdx.z * nrows + blockIdx.y) * NARR * M;
  const int n2_0 = blockIdx.x * NF;
  const int D = 1 << (log2L - LOGM);
  BandLoader<C, NARR, SIGN> ld{tb, zb, M, n2_0, log2L};
  typedef decltype(op.bind(0)) BOp;
  BandStore<BOp, C, SIGN> st{bop, tb, b, row, D, n2_0, klo, log2L};
  fft_rows<C, LOGM, NF, kNT, SIGN, NARR, MAP_J, MAP_F, true>(buf, seg_table<C>(tb), ld, st);
}

// shared memory of one tile kernel: NARR arrays of NF rows at the row pitch
template <typename C>
inline size_t tile_smem(int narr, int logl) {
  const int L = 1 << logl;
  const int NF = FftCfg<C>::TILE / L;
  const int G = 1 << FftCfg<C>::G_LOG;
  return (size_t)narr * NF * row_pitch(L, NF, G) * sizeof(C);
}

}  // namespace ssqb
