// Shared-memory Stockham FFT over a tile of NF independent sequences of
// length L = 2^LOGL (NF * L = TILE elements per array), NARR arrays
// transformed together (they share twiddles), radix 16/8/4/2 butterflies in
// registers. Stockham autosort formulation (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC 2008):
// stage with radix R after NS = prod(previous radices):
//   v[r] = x[j + r*L/R] * w_{NS*R}^{r*(j mod NS)},  v = DFT_R(v),
//   y[(j div NS)*NS*R + (j mod NS) + r*NS] = v[r].
// Each stage loads into registers, syncs, then stores in place.
#pragma once
#include "ssqb_common.cuh"

namespace ssqb {

// one spare slot per 16 elements: stride-R stores hit distinct banks
__host__ __device__ __forceinline__ constexpr int spad(int p) { return p + (p >> 4); }
__host__ __device__ constexpr int spad_size(int n) { return n + (n >> 4); }

// radix schedule for 2^m: radix-16 stages, finishing with 8 and/or 4
__host__ __device__ constexpr int fft_nstages(int m) {
  return m <= 4 ? 1 : (m % 4 == 0 ? m / 4 : m / 4 + 1);
}
__host__ __device__ constexpr int fft_rlog(int m, int s) {
  if (m <= 4) return m;
  int a = m / 4, r = m % 4;
  if (r == 0) return 4;
  if (r == 1) return s < a - 1 ? 4 : (s == a - 1 ? 3 : 2);
  if (r == 2) return s < a ? 4 : 2;
  return s < a ? 4 : 3;
}
__host__ __device__ constexpr int fft_lns(int m, int s) {
  int l = 0;
  for (int q = 0; q < s; ++q) l += fft_rlog(m, q);
  return l;
}

// cos / sin of a*pi/8
__host__ __device__ constexpr double cos16(int a) {
  constexpr double C1 = 0.92387953251128675613, C3 = 0.38268343236508977173,
                   H = 0.70710678118654752440;
  const double t[16] = {1.0, C1, H, C3, 0.0, -C3, -H, -C1,
                        -1.0, -C1, -H, -C3, 0.0, C3, H, C1};
  return t[a & 15];
}
__host__ __device__ constexpr double sin16(int a) { return cos16(a - 4); }

// v *= exp(SIGN*2*pi*i*a/16); `a` folds to a constant once loops unroll
template <int SIGN, typename C>
__device__ __forceinline__ C rot16(C v, int a) {
  typedef typename RealOf<C>::type T;
  a &= 15;
  if (a == 0) return v;
  if (a == 4) return cmul_i<SIGN>(v);
  if (a == 8) return mk(-v.x, -v.y);
  if (a == 12) return cmul_i<-SIGN>(v);
  const T c = (T)cos16(a);
  const T s = (T)(SIGN * sin16(a));
  return mk(v.x * c - v.y * s, v.x * s + v.y * c);
}

template <int R> __host__ __device__ constexpr int bitrev(int x) {
  int r = 0;
  for (int b = 1; b < R; b <<= 1) { r = (r << 1) | (x & 1); x >>= 1; }
  return r;
}

template <int R, int SIGN, typename C, int LEN>
__device__ __forceinline__ void dft_level(C (&v)[R]) {
  constexpr int half = LEN / 2;
#pragma unroll
  for (int b0 = 0; b0 < R; b0 += LEN) {
#pragma unroll
    for (int j = 0; j < half; ++j) {
      C u = v[b0 + j];
      C t = rot16<SIGN>(v[b0 + j + half], j * (16 / LEN));
      v[b0 + j] = cadd(u, t);
      v[b0 + j + half] = csub(u, t);
    }
  }
}

// In-register DFT of size R (2, 4, 8, 16), sign SIGN, natural order in/out.
template <int R, int SIGN, typename C>
__device__ __forceinline__ void dft(C (&v)[R]) {
  C t[R];
#pragma unroll
  for (int i = 0; i < R; ++i) t[i] = v[bitrev<R>(i)];
  if constexpr (R >= 2) dft_level<R, SIGN, C, 2>(t);
  if constexpr (R >= 4) dft_level<R, SIGN, C, 4>(t);
  if constexpr (R >= 8) dft_level<R, SIGN, C, 8>(t);
  if constexpr (R >= 16) dft_level<R, SIGN, C, 16>(t);
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = t[i];
}

template <typename C, int LOGL, int NF, int NT, int SIGN, int NARR, int S>
__device__ __forceinline__ void fft_stage(C* const (&buf)[NARR], const C* __restrict__ tw4k) {
  constexpr int L = 1 << LOGL;
  constexpr int RL = fft_rlog(LOGL, S);
  constexpr int R = 1 << RL;
  constexpr int LNS = fft_lns(LOGL, S);
  constexpr int NS = 1 << LNS;
  constexpr int NB = NF * L / R;
  constexpr int PER = (NB + NT - 1) / NT;
  constexpr int LR = LOGL - RL;  // log2(L/R)
  const int tid = threadIdx.x;
  C v[NARR][PER][R];
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int bb = tid + p * NT;
    if (NB % NT == 0 || bb < NB) {
      const int f = bb >> LR;
      const int j = bb & ((L / R) - 1);
#pragma unroll
      for (int a = 0; a < NARR; ++a)
#pragma unroll
        for (int r = 0; r < R; ++r) v[a][p][r] = buf[a][spad(f * L + j + r * (L / R))];
    }
  }
  __syncthreads();
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int bb = tid + p * NT;
    if (NB % NT == 0 || bb < NB) {
      const int f = bb >> LR;
      const int j = bb & ((L / R) - 1);
      const int k = j & (NS - 1);
      if constexpr (S > 0) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = __ldg(tw4k + ((r * k) << (12 - LNS - RL)));
          if (SIGN < 0) w.y = -w.y;
#pragma unroll
          for (int a = 0; a < NARR; ++a) v[a][p][r] = cmul(v[a][p][r], w);
        }
      }
#pragma unroll
      for (int a = 0; a < NARR; ++a) dft<R, SIGN>(v[a][p]);
      const int base = f * L + ((j >> LNS) << (LNS + RL)) + k;
#pragma unroll
      for (int a = 0; a < NARR; ++a)
#pragma unroll
        for (int r = 0; r < R; ++r) buf[a][spad(base + r * NS)] = v[a][p][r];
    }
  }
  __syncthreads();
}

// Full transform of the tile; caller must __syncthreads() after filling.
template <typename C, int LOGL, int NF, int NT, int SIGN, int NARR, int S = 0>
__device__ __forceinline__ void fft_tile(C* const (&buf)[NARR], const C* __restrict__ tw4k) {
  if constexpr (S < fft_nstages(LOGL)) {
    fft_stage<C, LOGL, NF, NT, SIGN, NARR, S>(buf, tw4k);
    fft_tile<C, LOGL, NF, NT, SIGN, NARR, S + 1>(buf, tw4k);
  }
}

}  // namespace ssqb
