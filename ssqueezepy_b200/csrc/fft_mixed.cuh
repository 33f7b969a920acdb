// Mixed-radix shared-memory Stockham FFT for transform lengths M that are a
// power of two times 5 (the chirp-z transform of an n_fft that is not a
// power of two needs M >= 2 n_fft - 1: M = 1280 = 5 * 4^4 instead of 2048 for
// n_fft 598). The same autosort stage as fft_tile.cuh with any radix
// R of a compile-time radix list:
//   v[r] = x[j + r*M/R] * w_{NS*R}^{r*(j mod NS)},  v = DFT_R(v),
//   y[(j div NS)*NS*R + (j mod NS) + r*NS] = v[r],  NS = product of the
// previous radices, w_{NS*R}^e = W[e * M/(NS*R)] from a table
// W[m] = exp(2 pi i m / M) in shared memory. One array, NF rows of M per
// CTA; inputs through the caller's loader, outputs left in shared memory.
//
// Shared-memory banks: a stage's twiddle reads step through the table at
// strides of 4, 16 or 64 entries, which a plain table puts on one 16-byte
// bank group (up to 8-way conflicts); tw_pos() XORs higher index bits into
// the bank-group bits. The data rows stay unswizzled: the stages' strides
// (1 and odd multiples within a quarter warp) are then nearly conflict free.
// Counted for M = 1280 (5, 4, 4, 4, 4) over a transform's accesses: 4,649
// wavefronts with a plain table and XOR-swizzled rows, 2,739 with these.
#pragma once
#include "fft_tile.cuh"

namespace ssqb {

template <int... Rs>
struct Radices {
  static constexpr int n = sizeof...(Rs);
  static constexpr int r[sizeof...(Rs)] = {Rs...};
  static constexpr int prod(int s) {
    int p = 1;
    for (int t = 0; t < s; ++t) p *= r[t];
    return p;
  }
};

// DFT of 5 points, sign SIGN, natural order (from the definition
// y_k = sum_n x_n e^{SIGN 2 pi i n k / 5}, sums and differences of the
// symmetric pairs first)
template <int SIGN, typename C>
__device__ __forceinline__ void dft5(C (&v)[5]) {
  typedef typename RealOf<C>::type T;
  const T c1 = (T)0.30901699437494742410;                // cos(2 pi / 5)
  const T c2 = (T)-0.80901699437494742410;               // cos(4 pi / 5)
  const T s1 = (T)(SIGN * 0.95105651629515357212);      // SIGN sin(2 pi / 5)
  const T s2 = (T)(SIGN * 0.58778525229247312917);      // SIGN sin(4 pi / 5)
  const C a1 = cadd(v[1], v[4]), d1 = csub(v[1], v[4]);
  const C a2 = cadd(v[2], v[3]), d2 = csub(v[2], v[3]);
  const C m1 = mk(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
  const C m2 = mk(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
  // i (s1 d1 + s2 d2) and i (s2 d1 - s1 d2)
  const C n1 = mk(-(s1 * d1.y + s2 * d2.y), s1 * d1.x + s2 * d2.x);
  const C n2 = mk(-(s2 * d1.y - s1 * d2.y), s2 * d1.x - s1 * d2.x);
  v[0] = cadd(v[0], cadd(a1, a2));
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

template <int R, int SIGN, typename C>
__device__ __forceinline__ void dft_any(C (&v)[R]) {
  if constexpr (R == 5) dft5<SIGN>(v);
  else dft<R, SIGN>(v);
}

// position of W[m] in the twiddle table (a permutation within each aligned
// group of 8 entries)
__device__ __forceinline__ int tw_pos(int m) { return m ^ (((m >> 3) ^ (m >> 6)) & 7); }

// rows of M at a pitch past M
template <typename C, int M, int NF>
struct LayoutM {
  static constexpr int G = 1 << FftCfg<C>::G_LOG;
  static constexpr int LP = M + (NF >= G ? 1 : (NF == 1 ? 0 : G / NF));
  static constexpr int ARR = NF * LP;
  __device__ __forceinline__ static int at(int f, int m) { return f * LP + m; }
};

template <typename C, int M, int NF, int NT, int SIGN, class RL, int S, class LD>
__device__ __forceinline__ void fft_mixed_stage(C* __restrict__ buf, const C* __restrict__ W,
                                                const LD& ld) {
  typedef LayoutM<C, M, NF> LY;
  constexpr int R = RL::r[S];
  constexpr int NS = RL::prod(S);
  constexpr int MR = M / R;
  constexpr int NB = NF * MR;
  constexpr int PER = cdiv(NB, NT);
  constexpr bool FIRST = (S == 0), LAST = (S == RL::n - 1);
  static_assert(M % R == 0, "radix must divide the length");
  const int tid = threadIdx.x;
  C v[PER][R];
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int it = tid + p * NT;
    if (NB % NT == 0 || it < NB) {
      const int f = it / MR, j = it % MR;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (FIRST) {
          C t[1];
          ld(f, j + r * MR, t);
          v[p][r] = t[0];
        } else {
          v[p][r] = buf[LY::at(f, j + r * MR)];
        }
      }
    }
  }
  if constexpr (!FIRST) __syncthreads();
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int it = tid + p * NT;
    if (NB % NT == 0 || it < NB) {
      const int f = it / MR, j = it % MR;
      const int k = j % NS;
      if constexpr (!FIRST) {
        constexpr int step = M / (NS * R);
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = W[tw_pos(r * k * step)];  // r k < NS R: the index stays below M
          if (SIGN < 0) w.y = -w.y;
          v[p][r] = cmul(v[p][r], w);
        }
      }
      dft_any<R, SIGN>(v[p]);
      const int base = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[LY::at(f, base + r * NS)] = v[p][r];
    }
  }
  __syncthreads();
  if constexpr (!LAST) fft_mixed_stage<C, M, NF, NT, SIGN, RL, S + 1>(buf, W, ld);
}

// One transform of NF rows of M; ld(f, m, C (&v)[1]) gives input m of row f
// and must not read `buf`. Outputs in natural order at LayoutM::at(f, n);
// ends with __syncthreads().
template <typename C, int M, int NF, int NT, int SIGN, class RL, class LD>
__device__ __forceinline__ void fft_mixed_rows(C* buf, const C* W, const LD& ld) {
  static_assert(RL::prod(RL::n) == M, "radices must multiply to the length");
  static_assert(M % 8 == 0, "tw_pos permutes aligned groups of 8 table entries");
  fft_mixed_stage<C, M, NF, NT, SIGN, RL, 0>(buf, W, ld);
}

}  // namespace ssqb
