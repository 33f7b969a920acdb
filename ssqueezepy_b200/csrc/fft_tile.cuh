// Shared-memory Stockham FFT over a tile of NF independent rows of length
// L = 2^LOGL, NARR arrays transformed together (they share twiddles and,
// at the ends, the prologue / epilogue), butterflies of radix <= RMAX in
// registers. Stockham autosort formulation (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC 2008):
// a stage of radix R after NS = product of the previous radices maps
//   v[r] = x[j + r*L/R] * w_{NS*R}^{r*(j mod NS)},  v = DFT_R(v),
//   y[(j div NS)*NS*R + (j mod NS) + r*NS] = v[r].
//
// The first stage reads its inputs straight from the caller's loader and the
// last stage (optionally) hands its outputs straight to the caller's storer,
// so only the L/R-strided exchanges between stages go through shared memory.
// Rows are XOR-swizzled in groups of G = 128 B / sizeof(C) elements and
// padded to a stride chosen so that both row-fastest and column-fastest
// thread mappings hit distinct banks.
#pragma once
#include <type_traits>
#include "ssqb_common.cuh"

namespace ssqb {

template <typename C> struct FftCfg;
template <> struct FftCfg<float2> {
  static constexpr int TILE = 4096, RMAX_LOG = 4, G_LOG = 4;
};
#ifndef SSQB_D_TILE
#define SSQB_D_TILE 2048
#endif
#ifndef SSQB_D_RLOG
#define SSQB_D_RLOG 3
#endif
template <> struct FftCfg<double2> {
  static constexpr int TILE = SSQB_D_TILE, RMAX_LOG = SSQB_D_RLOG, G_LOG = 3;
};

__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// radix schedule: ceil(m / RMAX_LOG) stages, radices as even as possible,
// larger ones first
__host__ __device__ constexpr int fft_nstages(int m, int rmax_log) {
  return m <= rmax_log ? 1 : cdiv(m, rmax_log);
}
__host__ __device__ constexpr int fft_rlog(int m, int rmax_log, int s) {
  const int n = fft_nstages(m, rmax_log);
  const int q = m / n, rem = m % n;
  return s < rem ? q + 1 : q;
}
__host__ __device__ constexpr int fft_lns(int m, int rmax_log, int s) {
  int l = 0;
  for (int t = 0; t < s; ++t) l += fft_rlog(m, rmax_log, t);
  return l;
}

// row stride: L plus an offset d so that f*LP covers distinct bank groups
// for f in [0, min(NF, G)) while the in-row swizzle handles the rest
__host__ __device__ constexpr int row_pitch(int L, int NF, int G) {
  return L + (NF >= G ? 1 : (NF == 1 ? 0 : G / NF));
}

template <typename C, int LOGL, int NF>
struct Layout {
  static constexpr int L = 1 << LOGL;
  static constexpr int G = 1 << FftCfg<C>::G_LOG;
  static constexpr int LP = row_pitch(L, NF, G);
  static constexpr int ARR = NF * LP;  // elements per array
  __device__ __forceinline__ static int at(int f, int m) {
    return f * LP + (m ^ ((m >> FftCfg<C>::G_LOG) & (G - 1)));
  }
};

// cos / sin of a*pi/16 (a in 0..31)
__host__ __device__ constexpr double cos32(int a) {
  const double t[32] = {
      1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
      0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173,
      0.19509032201612826785, 0.0, -0.19509032201612826785, -0.38268343236508977173,
      -0.55557023301960222474, -0.70710678118654752440, -0.83146961230254523708,
      -0.92387953251128675613, -0.98078528040323044913, -1.0, -0.98078528040323044913,
      -0.92387953251128675613, -0.83146961230254523708, -0.70710678118654752440,
      -0.55557023301960222474, -0.38268343236508977173, -0.19509032201612826785, 0.0,
      0.19509032201612826785, 0.38268343236508977173, 0.55557023301960222474,
      0.70710678118654752440, 0.83146961230254523708, 0.92387953251128675613,
      0.98078528040323044913};
  return t[a & 31];
}
__host__ __device__ constexpr double sin32(int a) { return cos32(a - 8); }

// v *= exp(SIGN*2*pi*i*a/32); `a` folds to a constant once loops unroll
template <int SIGN, typename C>
__device__ __forceinline__ C rot32(C v, int a) {
  typedef typename RealOf<C>::type T;
  a &= 31;
  if (a == 0) return v;
  if (a == 8) return cmul_i<SIGN>(v);
  if (a == 16) return mk(-v.x, -v.y);
  if (a == 24) return cmul_i<-SIGN>(v);
  const T c = (T)cos32(a);
  const T s = (T)(SIGN * sin32(a));
  return mk(v.x * c - v.y * s, v.x * s + v.y * c);
}

template <int R> __host__ __device__ constexpr int bitrev(int x) {
  int r = 0;
  for (int b = 1; b < R; b <<= 1) { r = (r << 1) | (x & 1); x >>= 1; }
  return r;
}

template <int R, int SIGN, int LEN, typename C>
__device__ __forceinline__ void dft_level(C (&t)[R]) {
  constexpr int half = LEN / 2;
#pragma unroll
  for (int b0 = 0; b0 < R; b0 += LEN) {
#pragma unroll
    for (int j = 0; j < half; ++j) {
      const C u = t[b0 + j];
      const C w = rot32<SIGN>(t[b0 + j + half], j * (32 / LEN));
      t[b0 + j] = cadd(u, w);
      t[b0 + j + half] = csub(u, w);
    }
  }
}

// In-register DFT of size R (2..16), sign SIGN, natural order in and out
// (radix-2 decimation in time over bit-reversed inputs).
template <int R, int SIGN, typename C>
__device__ __forceinline__ void dft(C (&v)[R]) {
  C t[R];
#pragma unroll
  for (int i = 0; i < R; ++i) t[i] = v[bitrev<R>(i)];
  if constexpr (R >= 2) dft_level<R, SIGN, 2>(t);
  if constexpr (R >= 4) dft_level<R, SIGN, 4>(t);
  if constexpr (R >= 8) dft_level<R, SIGN, 8>(t);
  if constexpr (R >= 16) dft_level<R, SIGN, 16>(t);
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = t[i];
}

// Thread mappings of butterfly items to (row f, column j in [0, L/R)).
enum { MAP_J = 0, MAP_F = 1 };
template <int MAP, int NF, int LR>
__device__ __forceinline__ void item_fj(int it, int& f, int& j) {
  if (MAP == MAP_J) { f = it >> LR; j = it & ((1 << LR) - 1); }
  else { f = it % NF; j = it / NF; }
}

// Twiddle segment table: seg[M + m] = exp(2 pi i m / M), M = 2..4096.
template <typename C> __device__ __forceinline__ const C* seg_table(const Tables& t);
template <> __device__ __forceinline__ const float2* seg_table<float2>(const Tables& t) {
  return t.seg_f;
}
template <> __device__ __forceinline__ const double2* seg_table<double2>(const Tables& t) {
  return t.seg_d;
}

// A loader with `kGather` gathers the R inputs of one first-stage item at
// once (`gather<R>(f, j, stride, t)`: inputs j + r*stride of row f), so that
// it can issue all of its memory loads before the arithmetic on them.
template <class T, class = void> struct HasGather : std::false_type {};
template <class T>
struct HasGather<T, std::void_t<decltype(T::kGather)>> : std::bool_constant<T::kGather> {};

// One full transform of the tile.
//   ld(f, m, C (&v)[NARR])   input element m of row f (all arrays)
//   st.item<R>(f, m0, stride, C (&a)[R], C (&b)[R])
//                            outputs m0 + r*stride of row f, r < R, of the
//                            first and last array (when DIRECT_OUT)
// buf: NARR arrays of Layout::ARR elements. MAP_IN / MAP_OUT: mappings of the
// first and last stage; middle stages use MAP_J. With DIRECT_OUT == false the
// last stage writes shared memory (read it back with Layout::at after the
// function returns; it ends with __syncthreads()).
template <typename C, int LOGL, int NF, int NT, int SIGN, int NARR, int MAP_IN, int MAP_OUT,
          bool DIRECT_OUT, int S, class LD, class ST>
__device__ __forceinline__ void fft_stage(C* const (&buf)[NARR], const C* __restrict__ seg,
                                          const LD& ld, const ST& st, int tid) {
  typedef Layout<C, LOGL, NF> LY;
  constexpr int RL_MAX = FftCfg<C>::RMAX_LOG;
  constexpr int NSTG = fft_nstages(LOGL, RL_MAX);
  constexpr int L = 1 << LOGL;
  constexpr int RL = fft_rlog(LOGL, RL_MAX, S);
  constexpr int R = 1 << RL;
  constexpr int LNS = fft_lns(LOGL, RL_MAX, S);
  constexpr int NS = 1 << LNS;
  constexpr int LR = LOGL - RL;
  constexpr int NB = NF * (L / R);
  constexpr int PER = cdiv(NB, NT);
  constexpr bool FIRST = (S == 0), LAST = (S == NSTG - 1);
  constexpr int MAP = FIRST ? MAP_IN : (LAST ? MAP_OUT : MAP_J);
  C v[NARR][PER][R];
  // gather
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int it = tid + p * NT;
    if (NB % NT == 0 || it < NB) {
      int f, j;
      item_fj<MAP, NF, LR>(it, f, j);
      if constexpr (FIRST && HasGather<LD>::value) {
        C t[R][NARR];
        ld.template gather<R>(f, j, L / R, t);
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int a = 0; a < NARR; ++a) v[a][p][r] = t[r][a];
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (FIRST && !HasGather<LD>::value) {
          C t[NARR];
          ld(f, j + r * (L / R), t);
#pragma unroll
          for (int a = 0; a < NARR; ++a) v[a][p][r] = t[a];
        } else if constexpr (!FIRST) {
#pragma unroll
          for (int a = 0; a < NARR; ++a) v[a][p][r] = buf[a][LY::at(f, j + r * (L / R))];
        }
      }
    }
  }
  if constexpr (!FIRST && !(LAST && DIRECT_OUT)) __syncthreads();
  // twiddle, butterfly, scatter
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int it = tid + p * NT;
    if (NB % NT == 0 || it < NB) {
      int f, j;
      item_fj<MAP, NF, LR>(it, f, j);
      const int k = j & (NS - 1);
      if constexpr (!FIRST) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = __ldg(seg + NS * R + r * k);
          if (SIGN < 0) w.y = -w.y;
#pragma unroll
          for (int a = 0; a < NARR; ++a) v[a][p][r] = cmul(v[a][p][r], w);
        }
      }
#pragma unroll
      for (int a = 0; a < NARR; ++a) dft<R, SIGN>(v[a][p]);
      const int base = ((j >> LNS) << (LNS + RL)) + k;
      if constexpr (LAST && DIRECT_OUT) {
        // outputs base + r*NS of row f, r = 0..R-1, handed over together
        st.template item<R>(f, base, NS, v[0][p], v[NARR - 1][p]);
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int a = 0; a < NARR; ++a) buf[a][LY::at(f, base + r * NS)] = v[a][p][r];
      }
    }
  }
  if constexpr (!(LAST && DIRECT_OUT)) __syncthreads();
  if constexpr (!LAST)
    fft_stage<C, LOGL, NF, NT, SIGN, NARR, MAP_IN, MAP_OUT, DIRECT_OUT, S + 1>(buf, seg, ld,
                                                                             st, tid);
}

// tid: this thread's index among the NT threads of the transform (a CTA can
// run several transforms side by side, each with its own NT threads; the
// stage barriers are CTA-wide, so all of them take the same stages)
template <typename C, int LOGL, int NF, int NT, int SIGN, int NARR, int MAP_IN, int MAP_OUT,
          bool DIRECT_OUT, class LD, class ST>
__device__ __forceinline__ void fft_rows(C* const (&buf)[NARR], const C* __restrict__ seg,
                                         const LD& ld, const ST& st, int tid = threadIdx.x) {
  fft_stage<C, LOGL, NF, NT, SIGN, NARR, MAP_IN, MAP_OUT, DIRECT_OUT, 0>(buf, seg, ld, st,
                                                                         tid);
}

}  // namespace ssqb
