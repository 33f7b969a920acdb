// Common device helpers: complex arithmetic, twiddle tables, status word.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ssqb {

template <typename T> struct CplxOf;
template <> struct CplxOf<float>  { typedef float2 type; };
template <> struct CplxOf<double> { typedef double2 type; };

template <typename C> struct RealOf;
template <> struct RealOf<float2>  { typedef float type; };
template <> struct RealOf<double2> { typedef double type; };

__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) {
  return mk(a.x * s, a.y * s);
}
// multiply by +i (sign > 0) or -i (sign < 0)
template <int SIGN, typename C> __device__ __forceinline__ C cmul_i(C a) {
  if (SIGN > 0) return mk(-a.y, a.x);
  return mk(a.y, -a.x);
}

template <typename C> __device__ __forceinline__ C to_c(double2 v);
template <> __device__ __forceinline__ float2 to_c<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
template <> __device__ __forceinline__ double2 to_c<double2>(double2 v) { return v; }

// Twiddle tables. The unit root exp(2*pi*i*e / 2^22) for e in [0, 2^22) is
// tw_hi[e >> 11] * tw_lo[e & 2047], both tables double precision (filled by
// sincospi in double on the device). seg_f / seg_d hold, for each power of
// two M = 2..4096, the M roots exp(2*pi*i*m/M) at [M, 2M), rounded once.
constexpr int TW_LOG = 22;
constexpr int TW_SPLIT = 11;
constexpr int SEG_SIZE = 8192;
struct Tables {
  const double2* tw_lo;   // 2048
  const double2* tw_hi;   // 2048
  const float2* seg_f;    // SEG_SIZE
  const double2* seg_d;   // SEG_SIZE
  int* status;            // device status word (0 = ok)
};

// exp(SIGN * 2*pi*i * e / 2^log2n), e in [0, 2^log2n), log2n <= 22, computed
// in double from the two-level table.
template <int SIGN>
__device__ __forceinline__ double2 unit_root(const Tables& t, uint32_t e, int log2n) {
  uint32_t E = e << (TW_LOG - log2n);
  double2 a = __ldg(t.tw_hi + (E >> TW_SPLIT));
  double2 b = __ldg(t.tw_lo + (E & ((1u << TW_SPLIT) - 1)));
  double2 r = mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  if (SIGN < 0) r.y = -r.y;
  return r;
}

// Status codes written to the device status word.
enum DeviceStatus : int {
  DEV_OK = 0,
  DEV_BAD_BIN = 1,      // a bin index fell outside [0, nbins)
  DEV_BAD_INDEX = 2,    // a padded-signal index fell outside the signal
  DEV_TIMEOUT = 3,      // a bounded wait on an asynchronous copy expired
};

__device__ __forceinline__ void set_status(int* st, int code) {
  if (st) atomicCAS(st, 0, code);
}

}  // namespace ssqb
