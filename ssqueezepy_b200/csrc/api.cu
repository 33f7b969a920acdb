// C-ABI layer: argument checks, per-device tables, dispatch to launchers.
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include "launch.h"
#include "../../include/ssqb.h"

namespace ssqb {

// Twiddle tables and the status word live in module memory (no cudaMalloc).
static __device__ double2 g_tw_lo[1 << TW_SPLIT];
static __device__ double2 g_tw_hi[1 << (TW_LOG - TW_SPLIT)];
static __device__ float2 g_seg_f[SEG_SIZE];
static __device__ double2 g_seg_d[SEG_SIZE];
static __device__ int g_status;

__global__ void init_tables_kernel() {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (1 << TW_SPLIT)) {  // exp(2 pi i t / 2^22)
    double s, c;
    sincospi((double)t / (double)(1 << (TW_LOG - 1)), &s, &c);
    g_tw_lo[t] = make_double2(c, s);
  }
  if (t < (1 << (TW_LOG - TW_SPLIT))) {  // exp(2 pi i t 2^11 / 2^22)
    double s, c;
    sincospi((double)t / (double)(1 << (TW_LOG - TW_SPLIT - 1)), &s, &c);
    g_tw_hi[t] = make_double2(c, s);
  }
  if (t >= 2 && t < SEG_SIZE) {  // segment M = 2^floor(log2 t): exp(2 pi i (t-M) / M)
    int M = 1;
    while ((M << 1) <= t) M <<= 1;
    double s, c;
    sincospi(2.0 * (double)(t - M) / (double)M, &s, &c);
    g_seg_d[t] = make_double2(c, s);
    g_seg_f[t] = make_float2((float)c, (float)s);
  }
  if (t == 0) g_status = 0;
}

static thread_local std::string t_err;
static std::mutex g_mu;
static bool g_init[256];
static Tables g_tables[256];

// Scratch of ssqb_cwt_noalloc: module memory, present on every device that
// loads this library until the process exits. Host code must not use the
// symbol's name as a device address; the address comes from
// cudaGetSymbolAddress, once per device (g_noalloc_ptr).
constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static void* g_noalloc_ptr[256];

static int fail(int code, const std::string& msg) {
  t_err = msg;
  return code;
}

static int cuda_fail(cudaError_t e, const char* where) {
  return fail(SSQB_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

static int get_tables(Tables* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 256) return fail(SSQB_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_init[dev]) {
    Tables t;
    void* p;
    if ((e = cudaGetSymbolAddress(&p, g_tw_lo))) return cuda_fail(e, "symbol tw_lo");
    t.tw_lo = (const double2*)p;
    if ((e = cudaGetSymbolAddress(&p, g_tw_hi))) return cuda_fail(e, "symbol tw_hi");
    t.tw_hi = (const double2*)p;
    if ((e = cudaGetSymbolAddress(&p, g_seg_f))) return cuda_fail(e, "symbol seg_f");
    t.seg_f = (const float2*)p;
    if ((e = cudaGetSymbolAddress(&p, g_seg_d))) return cuda_fail(e, "symbol seg_d");
    t.seg_d = (const double2*)p;
    if ((e = cudaGetSymbolAddress(&p, g_status))) return cuda_fail(e, "symbol status");
    t.status = (int*)p;
    init_tables_kernel<<<SEG_SIZE / 256, 256>>>();
    if ((e = cudaGetLastError())) return cuda_fail(e, "init tables");
    if ((e = cudaDeviceSynchronize())) return cuda_fail(e, "init tables sync");
    g_tables[dev] = t;
    g_init[dev] = true;
  }
  *out = g_tables[dev];
  return SSQB_OK;
}

static bool is_pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }
static int ilog2i(long long n) { int m = 0; while ((1LL << m) < n) ++m; return m; }

static int check_wavelet(const ssqb_wavelet* w, WavDev* out) {
  if (!w) return fail(SSQB_EINVAL, "wavelet is NULL");
  if (w->kind < 0 || w->kind > 2) return fail(SSQB_EINVAL, "unknown wavelet kind");
  out->kind = w->kind;
  out->p0 = w->p[0]; out->p1 = w->p[1]; out->p2 = w->p[2]; out->p3 = w->p[3];
  out->wcg = (w->kind == 1) ? std::pow(w->p[2], w->p[0]) : 0.0;
  out->lo = w->band[0];
  out->hi = w->band[1];
  out->ibeta = -1;
  if (w->kind == 1 && w->p[1] >= 0 && w->p[1] <= 128 && w->p[1] == std::floor(w->p[1]))
    out->ibeta = (int)w->p[1];
  if (w->kind != 0 && !(w->p[0] > 0 && w->p[1] > 0))
    return fail(SSQB_EINVAL, "GMW gamma and beta must be positive");
  if (w->npoly < 0 || w->npoly > 8)
    return fail(SSQB_EINVAL, "wavelet npoly must be in [0, 8]");
  if (w->npoly > 0 && w->kind == 0)
    return fail(SSQB_EINVAL, "wavelet npoly > 0 is for GMW kinds only");
  out->npoly = w->npoly;
  for (int m = 0; m < 8; ++m) {
    out->kc[m] = m < w->npoly ? w->kc[m] : 0.0;
    if (!std::isfinite(out->kc[m])) return fail(SSQB_EINVAL, "wavelet kc must be finite");
  }
  return SSQB_OK;
}

static int check_bins(const ssqb_bins* b, int na, BinDev* out) {
  if (!b) return fail(SSQB_EINVAL, "bins is NULL");
  if (b->mode < 0 || b->mode > 2) return fail(SSQB_EINVAL, "unknown bin mode");
  if (b->nbins < 1 || b->nbins > 65535)
    return fail(SSQB_EINVAL, "nbins must be in [1, 65535]");
  if (b->nbins != na) return fail(SSQB_EINVAL, "nbins must equal the number of rows");
  out->mode = b->mode; out->idx1 = b->idx1; out->flipud = b->flipud ? 1 : 0;
  out->nbins = b->nbins;
  out->p0 = b->p[0]; out->p1 = b->p[1]; out->p2 = b->p[2]; out->p3 = b->p[3];
  if (b->mode == 0 && !(b->p[1] > 0)) return fail(SSQB_EINVAL, "dvl must be > 0");
  if (b->mode == 1 && !(b->p[2] > 0 && b->p[3] > 0))
    return fail(SSQB_EINVAL, "dvl0, dvl1 must be > 0");
  if (b->mode == 2 && !(b->p[1] > 0)) return fail(SSQB_EINVAL, "dv must be > 0");
  return SSQB_OK;
}

// bytes of one complex value of the transform arithmetic
static size_t csize(int precision) { return precision == SSQB_F32 ? 8 : 16; }
static bool valid_precision(int p) { return p == SSQB_F32 || p == SSQB_F64 || p == SSQB_F32X; }
// storage precision of data arrays: F32X stores float32
static int data_prec(int p) { return p == SSQB_F32X ? SSQB_F32 : p; }

static size_t xhat_bytes(int B, int Npad) { return (size_t)B * Npad * sizeof(double2); }

static bool cwt_two_pass(int m, int precision) {
  return precision == SSQB_F32 ? two_pass<float2>(m) : two_pass<double2>(m);
}

// intermediate needed for one row: the float64 x_hat (if it takes two
// passes) and the CWT (if it does)
static size_t min_z_bytes(int B, int Npad, int precision) {
  const int m = ilog2i(Npad);
  const size_t a = two_pass<double2>(m) ? (size_t)B * Npad * sizeof(double2) : 0;
  const size_t c = cwt_two_pass(m, precision) ? (size_t)B * 2 * Npad * csize(precision) : 0;
  return a > c ? a : c;
}

// ---- batches of uneven lengths ------------------------------------------------
static_assert(sizeof(ssqb_sig) == sizeof(SigDesc), "ssqb_sig / SigDesc layout");
static_assert(offsetof(ssqb_sig, scales) == offsetof(SigDesc, scales), "ssqb_sig layout");
static_assert(offsetof(ssqb_sig, N) == offsetof(SigDesc, N), "ssqb_sig layout");
static_assert(offsetof(ssqb_sig, mode) == offsetof(SigDesc, mode), "ssqb_sig layout");
static_assert(offsetof(ssqb_sig, p) == offsetof(SigDesc, p0), "ssqb_sig layout");

// bound of the batch intermediate: chunks of signals and rows that fit it
constexpr size_t kBatchZBytes = (size_t)64 << 20;

static size_t batch_z_bytes(int Npad, int precision) {
  const size_t one = min_z_bytes(1, Npad, precision);
  return one == 0 ? 0 : (one > kBatchZBytes ? one : kBatchZBytes);
}

// host-side check of the descriptors; `Npad` > 0 also checks the padding
// geometry of each signal against it
static int check_sigs(const ssqb_sig* s, int nsig, int Npad, bool need_scales,
                      bool need_weights, int* max_na, int* max_N) {
  if (!s) return fail(SSQB_EINVAL, "sigs is NULL");
  if (nsig < 1 || nsig > 65535) return fail(SSQB_EINVAL, "nsig must be in [1, 65535]");
  int mna = 0, mN = 0;
  for (int i = 0; i < nsig; ++i) {
    const ssqb_sig& d = s[i];
    const std::string at = "signal " + std::to_string(i) + ": ";
    if (d.N < 1 || d.na < 1 || d.na > 65535)
      return fail(SSQB_EINVAL, at + "N must be >= 1 and na in [1, 65535]");
    if (d.x_off < 0 || d.out_off < 0 || d.idx_off < 0)
      return fail(SSQB_EINVAL, at + "negative offset");
    if (d.idx_pitch < d.N) return fail(SSQB_EINVAL, at + "idx_pitch smaller than N");
    if (Npad > 0 && (d.N > Npad || d.n1 < 0 || d.n1 + d.N > Npad))
      return fail(SSQB_EINVAL, at + "bad padding geometry");
    if (need_scales && !d.scales) return fail(SSQB_EINVAL, at + "scales is NULL");
    if (need_weights && !d.weights) return fail(SSQB_EINVAL, at + "weights is NULL");
    ssqb_bins b{d.mode, d.idx1, d.flipud, d.nbins, {d.p[0], d.p[1], d.p[2], d.p[3]}};
    BinDev bd;
    const int r = check_bins(&b, d.na, &bd);
    if (r) return fail(r, at + t_err);
    if (d.na > mna) mna = d.na;
    if (d.N > mN) mN = d.N;
  }
  *max_na = mna;
  *max_N = mN;
  return SSQB_OK;
}

// band rows: bands of at most TILE / 2^off bins (2^off residues per CTA of
// the single pass). With float64 arithmetic 1024 bins (off 1) measured
// fastest up to Npad = 65,536 and 512 (off 2) above (single calls at N =
// 10,000 / 60,000 / 160,000, and the batch autotuner's choices per length)
static int band_off(int Npad) { return Npad <= (1 << 16) ? 1 : 2; }
// Rows whose wavelet band fits at most 2^max_log bins, as band_bins
// evaluates it on the device (the same float64 expressions): the longest
// suffix of such rows takes the band-limited single pass. No host scales:
// every row takes the tile passes.
static void cwt_band_plan(const double* sc, int na, int Npad, const WavDev& wd, int max_log,
                          BandPlan* bp) {
  bp->two_pass_rows = na;
  bp->ngroups = 0;
  if (!sc || !(wd.lo < wd.hi)) return;
  const double h = (2 * M_PI) / Npad;
  std::vector<int> lg(na);
  for (int i = 0; i < na; ++i) {
    const double sh = sc[i] * h;
    const double a = std::floor(wd.lo / sh) - 1.0, c = std::ceil(wd.hi / sh) + 1.0;
    const int klo = (int)std::fmax(std::fmin(a, (double)Npad), -(double)Npad);
    const int khi = (int)std::fmax(std::fmin(c, (double)Npad), -(double)Npad);
    int l = 3;
    while ((1 << l) < khi - klo + 1) ++l;
    lg[i] = l;
  }
  int s = na;
  while (s > 0 && lg[s - 1] <= max_log) --s;
  if (s == na) return;
  // one group at the largest band length of the suffix: two launches in all
  // (per-length groups measured slower, their launches cost more than the
  // narrower transforms save)
  bp->two_pass_rows = s;
  bp->ngroups = 1;
  bp->r0[0] = s;
  bp->nrows[0] = na - s;
  bp->logM[0] = 3;
  for (int i = s; i < na; ++i)
    if (lg[i] > bp->logM[0]) bp->logM[0] = lg[i];
}

}  // namespace ssqb

using namespace ssqb;

extern "C" {

int ssqb_version(void) { return 1; }

const char* ssqb_last_error(void) { return t_err.c_str(); }

int ssqb_device_status(void* stream, int* status_out) {
  Tables tb;
  int r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, tb.status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (!e) e = cudaMemsetAsync(tb.status, 0, sizeof(int), st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) return cuda_fail(e, "device status");
  if (status_out) *status_out = h;
  return SSQB_OK;
}

size_t ssqb_cwt_workspace_bytes(int B, int N, int Npad, int na, int precision) {
  (void)N;
  if (B < 1 || Npad < 1 || na < 1) return 0;
  size_t z = min_z_bytes(B, Npad, precision);
  if (cwt_two_pass(ilog2i(Npad), precision)) {
    const size_t budget = cwt_z_budget(ilog2i(Npad));
    const size_t per_row = (size_t)B * 2 * Npad * csize(precision);
    size_t rows = budget / per_row;
    if (rows < 2) rows = 2;  // two row tiles, one per stream
    if (rows > (size_t)na) rows = na;
    z = rows * per_row;
    if (B > 1 && per_row > budget / 2) {
      // signals go in chunks whose two row tiles fit the budget
      const size_t per_sig = 2 * (size_t)Npad * csize(precision);
      size_t bc = budget / 2 / per_sig;
      if (bc < 1) bc = 1;
      z = 2 * bc * per_sig > budget ? 2 * bc * per_sig : budget;
    }
    const size_t mz = min_z_bytes(B, Npad, precision);
    if (z < mz) z = mz;
  }
  return xhat_bytes(B, Npad) + z;
}

static int cwt_launches_impl(int B, int Npad, int na, int precision, size_t workspace_bytes,
                             const BandPlan* bp) {
  if (B < 1 || na < 1 || !is_pow2(Npad) || Npad < 8 || Npad > (1 << 22)) return -1;
  if (!valid_precision(precision)) return -1;
  const size_t xb = xhat_bytes(B, Npad);
  if (workspace_bytes < xb + min_z_bytes(B, Npad, precision)) return -1;
  const size_t zbytes = workspace_bytes - xb;
  const int m = ilog2i(Npad);
  Tables tb{};
  int count = 0;
  set_launch_counter(&count);
  run_xhat_f32(nullptr, B, 1, Npad, 0, 1, nullptr, nullptr, zbytes / sizeof(double2), tb, 0);
  if (precision == SSQB_F32) {
    CwtOp<float2> op{};
    op.na = na;
    run_cwt_f32(op, B, m, nullptr, zbytes / sizeof(float2), tb, 0, bp);
  } else if (precision == SSQB_F32X) {
    CwtOp<double2, float2> op{};
    op.na = na;
    run_cwt_f32x(op, B, m, nullptr, zbytes / sizeof(double2), tb, 0, bp);
  } else {
    CwtOp<double2> op{};
    op.na = na;
    run_cwt_f64(op, B, m, nullptr, zbytes / sizeof(double2), tb, 0, bp);
  }
  set_launch_counter(nullptr);
  return count;
}

int ssqb_cwt_launches(int B, int Npad, int na, int precision, size_t workspace_bytes) {
  return cwt_launches_impl(B, Npad, na, precision, workspace_bytes, nullptr);
}

int ssqb_cwt_ex_launches(int B, int Npad, int na, int precision, size_t workspace_bytes,
                         const double* scales_host, const ssqb_wavelet* wavelet) {
  WavDev wd;
  if (!scales_host || check_wavelet(wavelet, &wd)) return -1;
  BandPlan bp{};
  const int max_log = ilog2i(precision == SSQB_F32 ? FftCfg<float2>::TILE
                                                  : FftCfg<double2>::TILE) - band_off(Npad);
  cwt_band_plan(scales_host, na, Npad, wd, max_log, &bp);
  return cwt_launches_impl(B, Npad, na, precision, workspace_bytes, &bp);
}

static int cwt_impl(const void* x, int B, int N, int Npad, int n1, int padtype, int rpadded,
                    const double* scales, int na, const ssqb_wavelet* wavelet, double dt,
                    const ssqb_bins* bins, double gamma, int precision,
                    void* Wx, void* dWx, void* w, uint16_t* idx, int idx_pitch,
                    void* workspace, size_t workspace_bytes, void* stream,
                    const double* scales_host) {
  if (!x || !scales || !Wx || !workspace) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || N < 1 || na < 1) return fail(SSQB_EINVAL, "B, N and na must be >= 1");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  if (!is_pow2(Npad) || Npad < 8 || Npad > (1 << 22))
    return fail(SSQB_EUNSUPPORTED, "Npad must be a power of two in [8, 2^22]");
  if (Npad < N || n1 < 0 || n1 + N > Npad) return fail(SSQB_EINVAL, "bad padding geometry");
  if (padtype < 0 || padtype > 5) return fail(SSQB_EINVAL, "unknown padtype");
  if (!(dt > 0)) return fail(SSQB_EINVAL, "dt must be > 0");
  if (B > 65535 || na > 65535) return fail(SSQB_EINVAL, "B and na must be <= 65535");
  WavDev wd;
  int r = check_wavelet(wavelet, &wd);
  if (r) return r;
  BinDev bd{};
  if (idx) {
    r = check_bins(bins, na, &bd);
    if (r) return r;
  }
  if (idx_pitch == 0) idx_pitch = rpadded ? Npad : N;
  if (idx && idx_pitch < (rpadded ? Npad : N))
    return fail(SSQB_EINVAL, "idx_pitch smaller than the row length");
  const size_t need = xhat_bytes(B, Npad) + min_z_bytes(B, Npad, precision);
  if (workspace_bytes < need)
    return fail(SSQB_EWORKSPACE, "workspace too small: need " + std::to_string(need) +
                                     " bytes");
  Tables tb;
  r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  double2* xh = (double2*)workspace;
  unsigned char* zb = (unsigned char*)workspace + xhat_bytes(B, Npad);
  const size_t zbytes = workspace_bytes - xhat_bytes(B, Npad);
  int e;
  if (data_prec(precision) == SSQB_F32)
    e = run_xhat_f32((const float*)x, B, N, Npad, n1, padtype, xh, (double2*)zb,
                     zbytes / sizeof(double2), tb, st);
  else
    e = run_xhat_f64((const double*)x, B, N, Npad, n1, padtype, xh, (double2*)zb,
                     zbytes / sizeof(double2), tb, st);
  if (e) return cuda_fail((cudaError_t)e, "x_hat launch");
  const int m = ilog2i(Npad);
  const double h = (2 * M_PI) / Npad;
  const int oN = rpadded ? Npad : N, on1 = rpadded ? 0 : n1;
  BandPlan bp{};
  const int max_log = ilog2i(precision == SSQB_F32 ? FftCfg<float2>::TILE
                                                  : FftCfg<double2>::TILE) - band_off(Npad);
  cwt_band_plan(scales_host, na, Npad, wd, max_log, &bp);
  if (precision == SSQB_F32) {
    CwtOp<float2> op{xh, scales, wd, bd, na, oN, Npad, on1, h, 1.0 / dt,
                     (float)(1.0 / Npad), gamma, (float2*)Wx, (float2*)dWx, (float*)w,
                     idx, idx_pitch, tb.status};
    e = run_cwt_f32(op, B, m, (float2*)zb, zbytes / sizeof(float2), tb, st, &bp);
  } else if (precision == SSQB_F32X) {
    CwtOp<double2, float2> op{xh, scales, wd, bd, na, oN, Npad, on1, h, 1.0 / dt,
                              1.0 / Npad, gamma, (float2*)Wx, (float2*)dWx, (float*)w,
                              idx, idx_pitch, tb.status};
    e = run_cwt_f32x(op, B, m, (double2*)zb, zbytes / sizeof(double2), tb, st, &bp);
  } else {
    CwtOp<double2> op{xh, scales, wd, bd, na, oN, Npad, on1, h, 1.0 / dt, 1.0 / Npad,
                      gamma, (double2*)Wx, (double2*)dWx, (double*)w, idx, idx_pitch,
                      tb.status};
    e = run_cwt_f64(op, B, m, (double2*)zb, zbytes / sizeof(double2), tb, st, &bp);
  }
  if (e) return cuda_fail((cudaError_t)e, "cwt launch");
  return SSQB_OK;
}

int ssqb_cwt(const void* x, int B, int N, int Npad, int n1, int padtype, int rpadded,
             const double* scales, int na, const ssqb_wavelet* wavelet, double dt,
             const ssqb_bins* bins, double gamma, int precision,
             void* Wx, void* dWx, void* w, uint16_t* idx, int idx_pitch,
             void* workspace, size_t workspace_bytes, void* stream) {
  return cwt_impl(x, B, N, Npad, n1, padtype, rpadded, scales, na, wavelet, dt, bins, gamma,
                  precision, Wx, dWx, w, idx, idx_pitch, workspace, workspace_bytes, stream,
                  nullptr);
}

int ssqb_cwt_ex(const void* x, int B, int N, int Npad, int n1, int padtype, int rpadded,
                const double* scales, const double* scales_host, int na,
                const ssqb_wavelet* wavelet, double dt, const ssqb_bins* bins, double gamma,
                int precision, void* Wx, void* dWx, void* w, uint16_t* idx, int idx_pitch,
                void* workspace, size_t workspace_bytes, void* stream) {
  return cwt_impl(x, B, N, Npad, n1, padtype, rpadded, scales, na, wavelet, dt, bins, gamma,
                  precision, Wx, dWx, w, idx, idx_pitch, workspace, workspace_bytes, stream,
                  scales_host);
}

static int squeeze_common(const void* Wx, int kind, const void* src, int idx_pitch,
                          const double* sfs, const double* cst, const ssqb_bins* bins,
                          double gamma, int B, int na, int N, int nbins, int precision,
                          void* Tx, void* stream) {
  if (!Wx || !src || !cst || !Tx) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || N < 1 || na < 1) return fail(SSQB_EINVAL, "B, N and na must be >= 1");
  if (B > 65535) return fail(SSQB_EINVAL, "B must be <= 65535");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  precision = data_prec(precision);
  if (nbins < 1 || nbins > 65535) return fail(SSQB_EINVAL, "nbins must be in [1, 65535]");
  if (idx_pitch == 0) idx_pitch = N;
  if (kind == 0 && idx_pitch < N) return fail(SSQB_EINVAL, "idx_pitch smaller than N");
  BinDev bd{};
  if (kind != 0) {
    int r = check_bins(bins, nbins, &bd);
    if (r) return r;
  }
  const size_t smem = (size_t)nbins * 8 * csize(precision) +
                      (size_t)na * (precision == SSQB_F64 ? 8 : 4);  // 8 columns per warp
  if (smem > 227 * 1024)
    return fail(SSQB_EUNSUPPORTED, "too many bins for the shared-memory squeeze");
  Tables tb;
  int r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  int e;
  if (precision == SSQB_F32)
    e = run_squeeze_f32((const float2*)Wx, kind, src, idx_pitch, sfs, bd, gamma, cst, B, na,
                        N, nbins, (float2*)Tx, tb.status, st);
  else
    e = run_squeeze_f64((const double2*)Wx, kind, src, idx_pitch, sfs, bd, gamma, cst, B, na,
                        N, nbins, (double2*)Tx, tb.status, st);
  if (e) return cuda_fail((cudaError_t)e, "squeeze launch");
  return SSQB_OK;
}

int ssqb_squeeze(const void* Wx, const uint16_t* idx, int idx_pitch,
                 const double* row_weights, int B, int na, int N, int nbins, int precision,
                 void* Tx, void* stream) {
  return squeeze_common(Wx, 0, idx, idx_pitch, nullptr, row_weights, nullptr, 0.0, B, na, N,
                        nbins, precision, Tx, stream);
}

int ssqb_ssqueeze_fast(const void* Wx, const void* dWx, const double* Sfs,
                       const double* row_weights, const ssqb_bins* bins, double gamma,
                       int B, int na, int N, int precision, void* Tx, void* stream) {
  return squeeze_common(Wx, 1, dWx, 0, Sfs, row_weights, bins, gamma, B, na, N,
                        bins ? bins->nbins : 0, precision, Tx, stream);
}

int ssqb_indexed_sum(const void* Wx, const void* w, const double* row_weights,
                     const ssqb_bins* bins, int B, int na, int N, int precision, void* Tx,
                     void* stream) {
  return squeeze_common(Wx, 2, w, 0, nullptr, row_weights, bins, 0.0, B, na, N,
                        bins ? bins->nbins : 0, precision, Tx, stream);
}

int ssqb_stft(const void* x, int B, int N, int n_fft, int hop, int n1, int padtype,
              int modulated, const double* window, const double* diff_window,
              const double* Sfs, const ssqb_bins* bins, double gamma, int precision,
              void* Sx, void* dSx, void* w, uint16_t* idx, int idx_pitch, void* stream) {
  if (!x || !window || !diff_window || !Sfs || !Sx)
    return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || N < 1 || hop < 1) return fail(SSQB_EINVAL, "B, N and hop must be >= 1");
  if (B > 65535) return fail(SSQB_EINVAL, "B must be <= 65535");
  const bool pow2 = is_pow2(n_fft);
  // other lengths go through Bluestein's transform of length M >= 2 n_fft - 1,
  // which must fit one float64 tile
  int log2M = 0;
  while ((1 << log2M) < 2 * n_fft - 1) ++log2M;
  if (pow2 ? (n_fft < 8 || n_fft > 4096)
           : (n_fft < 4 || (1 << log2M) > FftCfg<double2>::TILE))
    return fail(SSQB_EUNSUPPORTED,
                "n_fft must be a power of two in [8, 4096] or any length in [4, " +
                    std::to_string((FftCfg<double2>::TILE + 1) / 2) + "]");
  if (padtype < 0 || padtype > 5) return fail(SSQB_EINVAL, "unknown padtype");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  if (pow2 && precision != SSQB_F32 && n_fft > FftCfg<double2>::TILE)
    return fail(SSQB_EUNSUPPORTED, "n_fft above " + std::to_string(FftCfg<double2>::TILE) +
                                       " needs float32 arithmetic");
  const int nrow = n_fft / 2 + 1;
  const int nframes = (N - 1) / hop + 1;
  if (idx_pitch == 0) idx_pitch = nframes;
  if (idx && idx_pitch < nframes) return fail(SSQB_EINVAL, "idx_pitch smaller than n_frames");
  BinDev bd{};
  if (idx) {
    int r = check_bins(bins, nrow, &bd);
    if (r) return r;
  }
  Tables tb;
  int r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  const int s20 = (n_fft + 1) / 2;
  const int s21 = (n_fft % 2 == 1) ? s20 - 1 : s20;
  const int m = ilog2i(n_fft);
  int e;
  if (!pow2) {
    if (data_prec(precision) == SSQB_F64) {
      StftOp<double, double2> op{(const double*)x, window, diff_window, Sfs, bd, N, n_fft,
                                 hop, n1, padtype, s21, modulated ? 1 : 0, nframes, gamma,
                                 (double2*)Sx, (double2*)dSx, (double*)w, idx, idx_pitch,
                                 tb.status};
      e = run_stft_any_f64(op, B, log2M, tb, st);
    } else {
      StftOp<float, double2, float2> op{(const float*)x, window, diff_window, Sfs, bd, N,
                                        n_fft, hop, n1, padtype, s21, modulated ? 1 : 0,
                                        nframes, gamma, (float2*)Sx, (float2*)dSx,
                                        (float*)w, idx, idx_pitch, tb.status};
      e = run_stft_any_f32x(op, B, log2M, tb, st);
    }
  } else if (precision == SSQB_F32) {
    StftOp<float, float2> op{(const float*)x, window, diff_window, Sfs, bd, N, n_fft, hop,
                             n1, padtype, s21, modulated ? 1 : 0, nframes, gamma,
                             (float2*)Sx, (float2*)dSx, (float*)w, idx, idx_pitch, tb.status};
    e = run_stft_f32(op, B, m, tb, st);
  } else if (precision == SSQB_F32X) {
    StftOp<float, double2, float2> op{(const float*)x, window, diff_window, Sfs, bd, N,
                                      n_fft, hop, n1, padtype, s21, modulated ? 1 : 0,
                                      nframes, gamma, (float2*)Sx, (float2*)dSx, (float*)w,
                                      idx, idx_pitch, tb.status};
    e = run_stft_f32x(op, B, m, tb, st);
  } else {
    StftOp<double, double2> op{(const double*)x, window, diff_window, Sfs, bd, N, n_fft,
                               hop, n1, padtype, s21, modulated ? 1 : 0, nframes, gamma,
                               (double2*)Sx, (double2*)dSx, (double*)w, idx, idx_pitch,
                               tb.status};
    e = run_stft_f64(op, B, m, tb, st);
  }
  if (e) return cuda_fail((cudaError_t)e, "stft launch");
  return SSQB_OK;
}

int ssqb_icwt(const void* Wx, const double* row_weights, const double* x_mean,
              double mean_weight, int B, int na, int N, int precision, void* x,
              void* stream) {
  if (!Wx || !row_weights || !x) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || N < 1 || na < 1) return fail(SSQB_EINVAL, "B, N and na must be >= 1");
  if (B > 65535) return fail(SSQB_EINVAL, "B must be <= 65535");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  precision = data_prec(precision);
  int e = run_icwt(Wx, row_weights, x_mean, mean_weight, B, na, N, precision, x,
                   (cudaStream_t)stream);
  if (e) return cuda_fail((cudaError_t)e, "icwt launch");
  return SSQB_OK;
}

int ssqb_issq(const void* Tx, int nrows, int N, const int32_t* cc, const int32_t* cw, int K,
              double scale, int precision, void* x, void* stream) {
  if (!Tx || !x) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (nrows < 1 || N < 1) return fail(SSQB_EINVAL, "nrows and N must be >= 1");
  if (K < 0 || K > 16) return fail(SSQB_EUNSUPPORTED, "K must be in [0, 16]");
  if (K > 0 && (!cc || !cw)) return fail(SSQB_EINVAL, "components need cc and cw");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  const int e = run_issq(Tx, nrows, N, cc, cw, K, scale, data_prec(precision), x,
                         (cudaStream_t)stream);
  if (e) return cuda_fail((cudaError_t)e, "issq launch");
  return SSQB_OK;
}

size_t ssqb_ridges_workspace_bytes(int nf, int N, int precision) {
  if (nf < 1 || N < 1 || !valid_precision(precision)) return 0;
  return ridges_workspace(nf, N, data_prec(precision) == SSQB_F64);
}

int ssqb_extract_ridges(const void* Tf, int nf, int N, const void* s, const void* scales,
                        double penalty, int n_ridges, int bw, double eps, int precision,
                        int32_t* ridge_idx, void* ridge_f, void* ridge_e, void* workspace,
                        size_t workspace_bytes, void* stream) {
  if (!Tf || !s || !scales || !ridge_idx || !workspace)
    return fail(SSQB_EINVAL, "NULL pointer argument");
  if (nf < 1 || N < 1 || n_ridges < 1) return fail(SSQB_EINVAL, "nf, N, n_ridges must be >= 1");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  const bool f64 = data_prec(precision) == SSQB_F64;
  if (2 * (size_t)nf * (f64 ? 8 : 4) > 227 * 1024)
    return fail(SSQB_EUNSUPPORTED, "too many frequency rows for the shared-memory sweep");
  const size_t need = ridges_workspace(nf, N, f64);
  if (workspace_bytes < need)
    return fail(SSQB_EWORKSPACE, "workspace too small: need " + std::to_string(need) +
                                     " bytes");
  const int e = run_ridges(Tf, nf, N, s, scales, penalty, n_ridges, bw, eps, f64, ridge_idx,
                           ridge_f, ridge_e, workspace, (cudaStream_t)stream);
  if (e) return cuda_fail((cudaError_t)e, "ridge launch");
  return SSQB_OK;
}

int ssqb_cwt_noalloc(const void* x, int B, int N, int Npad, int n1, int padtype,
                     int rpadded, const double* scales, int na,
                     const ssqb_wavelet* wavelet, double dt, const ssqb_bins* bins,
                     double gamma, int precision, void* Wx, void* dWx, void* w,
                     uint16_t* idx, int idx_pitch, void* stream) {
  // the checks that size the scratch come first, with ssqb_cwt's codes and
  // messages; ssqb_cwt repeats all of its checks on the call below
  if (B < 1 || N < 1 || na < 1) return fail(SSQB_EINVAL, "B, N and na must be >= 1");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  if (!is_pow2(Npad) || Npad < 8 || Npad > (1 << 22))
    return fail(SSQB_EUNSUPPORTED, "Npad must be a power of two in [8, 2^22]");
  if (B > 65535 || na > 65535) return fail(SSQB_EINVAL, "B and na must be <= 65535");
  const size_t need = xhat_bytes(B, Npad) + min_z_bytes(B, Npad, precision);
  if (need > kNoAllocScratchBytes)
    return fail(SSQB_EINVAL,
                "ssqb_cwt_noalloc: this call needs " + std::to_string(need) +
                    " bytes of scratch, more than its fixed " +
                    std::to_string(kNoAllocScratchBytes) +
                    " bytes; use ssqb_cwt with a caller workspace");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 256) return fail(SSQB_EINVAL, "device ordinal out of range");
  void* scratch;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      if ((e = cudaGetSymbolAddress(&p, g_noalloc_scratch)))
        return cuda_fail(e, "symbol noalloc scratch");
      g_noalloc_ptr[dev] = p;
    }
    scratch = g_noalloc_ptr[dev];
  }
  // one stream only: this entry point creates no stream or event either
  set_aux_streams(false);
  const int r = ssqb_cwt(x, B, N, Npad, n1, padtype, rpadded, scales, na, wavelet, dt, bins,
                         gamma, precision, Wx, dWx, w, idx, idx_pitch, scratch,
                         kNoAllocScratchBytes, stream);
  set_aux_streams(true);
  return r;
}

size_t ssqb_cwt_noalloc_max_bytes(void) { return kNoAllocScratchBytes; }

size_t ssqb_cwt_batch_workspace_bytes(int nsig, int Npad, int precision) {
  if (nsig < 1 || !is_pow2(Npad)) return 0;
  return xhat_bytes(nsig, Npad) + batch_z_bytes(Npad, precision);
}

// band rows: at most half a tile of bins (at least two residues per CTA)
static int band_log_max(int precision) {
  return ilog2i(precision == SSQB_F32 ? FftCfg<float2>::TILE : FftCfg<double2>::TILE) - 1;
}

static int cwt_batch_impl(const float* x, const ssqb_sig* sigs, const ssqb_sig* sigs_dev,
                          int nsig, int Npad, int padtype, const ssqb_wavelet* wavelet,
                          double dt, double gamma, int precision, void* Wx, uint16_t* idx,
                          void* workspace, size_t workspace_bytes, int band_from,
                          int band_log, void* stream) {
  if (!x || !sigs_dev || !Wx || !idx || !workspace)
    return fail(SSQB_EINVAL, "NULL pointer argument");
  if (precision != SSQB_F32 && precision != SSQB_F32X)
    return fail(SSQB_EUNSUPPORTED, "batches take float32 data: precision SSQB_F32 or SSQB_F32X");
  if (!is_pow2(Npad) || Npad < 8 || Npad > (1 << 22))
    return fail(SSQB_EUNSUPPORTED, "Npad must be a power of two in [8, 2^22]");
  if (padtype < 0 || padtype > 5) return fail(SSQB_EINVAL, "unknown padtype");
  if (!(dt > 0)) return fail(SSQB_EINVAL, "dt must be > 0");
  int max_na = 0, max_N = 0;
  int r = check_sigs(sigs, nsig, Npad, true, false, &max_na, &max_N);
  if (r) return r;
  WavDev wd;
  r = check_wavelet(wavelet, &wd);
  if (r) return r;
  if (band_from < 0) return fail(SSQB_EINVAL, "band_from must be >= 0");
  if (band_from < max_na && (band_log < 3 || band_log > band_log_max(precision)))
    return fail(SSQB_EINVAL, "band_log must be in [3, " +
                                 std::to_string(band_log_max(precision)) + "]");
  const size_t xb = xhat_bytes(nsig, Npad);
  const size_t need = xb + min_z_bytes(1, Npad, precision);
  if (workspace_bytes < need)
    return fail(SSQB_EWORKSPACE, "workspace too small: need " + std::to_string(need) +
                                     " bytes");
  Tables tb;
  r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  const SigDesc* dd = reinterpret_cast<const SigDesc*>(sigs_dev);
  double2* xh = (double2*)workspace;
  unsigned char* zb = (unsigned char*)workspace + xb;
  const size_t zbytes = workspace_bytes - xb;
  int e = run_xhat_batch_f32(x, dd, nsig, Npad, padtype, xh, (double2*)zb,
                             zbytes / sizeof(double2), tb, st);
  if (e) return cuda_fail((cudaError_t)e, "x_hat launch");
  const int m = ilog2i(Npad);
  const double h = (2 * M_PI) / Npad;
  if (precision == SSQB_F32X) {
    CwtBatchOp<double2, float2> op{xh, dd, wd, Npad, h, 1.0 / dt, 1.0 / Npad, gamma,
                                   (float2*)Wx, idx, tb.status};
    op.band_from = band_from;
    e = run_cwt_batch_f32x(op, nsig, max_na, m, band_log, (double2*)zb,
                           zbytes / sizeof(double2), tb, st);
  } else {
    CwtBatchOp<float2, float2> op{xh, dd, wd, Npad, h, 1.0 / dt, (float)(1.0 / Npad), gamma,
                                  (float2*)Wx, idx, tb.status};
    op.band_from = band_from;
    e = run_cwt_batch_f32(op, nsig, max_na, m, band_log, (float2*)zb,
                          zbytes / sizeof(float2), tb, st);
  }
  if (e) return cuda_fail((cudaError_t)e, "cwt launch");
  return SSQB_OK;
}

int ssqb_cwt_batch(const float* x, const ssqb_sig* sigs, const ssqb_sig* sigs_dev, int nsig,
                   int Npad, int padtype, const ssqb_wavelet* wavelet, double dt,
                   double gamma, int precision, void* Wx, uint16_t* idx, void* workspace,
                   size_t workspace_bytes, void* stream) {
  return cwt_batch_impl(x, sigs, sigs_dev, nsig, Npad, padtype, wavelet, dt, gamma,
                        precision, Wx, idx, workspace, workspace_bytes, 0x7fffffff, 0, stream);
}

int ssqb_cwt_batch_ex(const float* x, const ssqb_sig* sigs, const ssqb_sig* sigs_dev,
                      int nsig, int Npad, int padtype, const ssqb_wavelet* wavelet, double dt,
                      double gamma, int precision, void* Wx, uint16_t* idx, void* workspace,
                      size_t workspace_bytes, int band_from, int band_log, void* stream) {
  return cwt_batch_impl(x, sigs, sigs_dev, nsig, Npad, padtype, wavelet, dt, gamma,
                        precision, Wx, idx, workspace, workspace_bytes, band_from, band_log,
                        stream);
}

int ssqb_cwt_band_rows(const double* scales_host, int na, int Npad,
                       const ssqb_wavelet* wavelet, int precision, int max_bins,
                       int* band_from, int* band_log) {
  if (!scales_host || !band_from || !band_log) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (na < 1 || !is_pow2(Npad) || Npad < 8 || Npad > (1 << 22))
    return fail(SSQB_EINVAL, "na must be >= 1 and Npad a power of two in [8, 2^22]");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  WavDev wd;
  int r = check_wavelet(wavelet, &wd);
  if (r) return r;
  int max_log = ilog2i(precision == SSQB_F32 ? FftCfg<float2>::TILE
                                             : FftCfg<double2>::TILE) - band_off(Npad);
  if (max_bins > 0) {
    if (!is_pow2(max_bins) || ilog2i(max_bins) > band_log_max(precision))
      return fail(SSQB_EINVAL, "max_bins must be a power of two of at most half a tile");
    max_log = ilog2i(max_bins);
  }
  BandPlan bp{};
  cwt_band_plan(scales_host, na, Npad, wd, max_log, &bp);
  *band_from = bp.two_pass_rows;
  *band_log = bp.ngroups ? bp.logM[0] : 0;
  return SSQB_OK;
}

static int cwt_batch_launches_impl(const ssqb_sig* sigs, int nsig, int Npad, int precision,
                                   size_t workspace_bytes, int band_from, int band_log) {
  if (precision != SSQB_F32 && precision != SSQB_F32X) return -1;
  if (!is_pow2(Npad) || Npad < 8 || Npad > (1 << 22)) return -1;
  int max_na = 0, max_N = 0;
  if (check_sigs(sigs, nsig, Npad, false, false, &max_na, &max_N)) return -1;
  const size_t xb = xhat_bytes(nsig, Npad);
  if (workspace_bytes < xb + min_z_bytes(1, Npad, precision)) return -1;
  const size_t zbytes = workspace_bytes - xb;
  Tables tb{};
  int count = 0;
  set_launch_counter(&count);
  run_xhat_batch_f32(nullptr, nullptr, nsig, Npad, 1, nullptr, nullptr,
                     zbytes / sizeof(double2), tb, 0);
  const int m = ilog2i(Npad);
  if (precision == SSQB_F32X) {
    CwtBatchOp<double2, float2> op{};
    op.band_from = band_from;
    run_cwt_batch_f32x(op, nsig, max_na, m, band_log, nullptr, zbytes / sizeof(double2), tb,
                       0);
  } else {
    CwtBatchOp<float2, float2> op{};
    op.band_from = band_from;
    run_cwt_batch_f32(op, nsig, max_na, m, band_log, nullptr, zbytes / sizeof(float2), tb, 0);
  }
  set_launch_counter(nullptr);
  return count;
}

int ssqb_cwt_batch_launches(const ssqb_sig* sigs, int nsig, int Npad, int precision,
                            size_t workspace_bytes) {
  return cwt_batch_launches_impl(sigs, nsig, Npad, precision, workspace_bytes, 0x7fffffff, 0);
}

int ssqb_cwt_batch_ex_launches(const ssqb_sig* sigs, int nsig, int Npad, int precision,
                               size_t workspace_bytes, int band_from, int band_log) {
  if (band_from < 0 || band_log < 0 || band_log > band_log_max(precision)) return -1;
  return cwt_batch_launches_impl(sigs, nsig, Npad, precision, workspace_bytes, band_from,
                                 band_log);
}

int ssqb_squeeze_batch(const void* Wx, const uint16_t* idx, const ssqb_sig* sigs,
                       const ssqb_sig* sigs_dev, int nsig, int precision, void* Tx,
                       void* stream) {
  if (!Wx || !idx || !sigs_dev || !Tx) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (precision != SSQB_F32 && precision != SSQB_F32X)
    return fail(SSQB_EUNSUPPORTED, "batches take float32 data: precision SSQB_F32 or SSQB_F32X");
  int max_na = 0, max_N = 0;
  int r = check_sigs(sigs, nsig, 0, false, true, &max_na, &max_N);
  if (r) return r;
  const size_t smem = (size_t)max_na * 8 * sizeof(float2) + (size_t)max_na * sizeof(float);
  if (smem > 227 * 1024)
    return fail(SSQB_EUNSUPPORTED, "too many bins for the shared-memory squeeze");
  Tables tb;
  r = get_tables(&tb);
  if (r) return r;
  int e = run_squeeze_batch_f32((const float2*)Wx, idx,
                                reinterpret_cast<const SigDesc*>(sigs_dev), nsig, max_na,
                                max_N, (float2*)Tx, tb.status, (cudaStream_t)stream);
  if (e) return cuda_fail((cudaError_t)e, "squeeze launch");
  return SSQB_OK;
}

// ---- adjoints ------------------------------------------------------------------
static int check_adj_sources(const void* gWx, const void* gTx, const uint16_t* idx,
                             int idx_pitch, const double* sq_weights, int nbins,
                             const void* gxr, const double* icwt_weights, int N) {
  if (!gWx && !gTx && !gxr) return fail(SSQB_EINVAL, "no gradient source given");
  if (gTx) {
    if (!idx || !sq_weights) return fail(SSQB_EINVAL, "gTx needs idx and sq_weights");
    if (nbins < 1 || nbins > 65535) return fail(SSQB_EINVAL, "nbins must be in [1, 65535]");
    if (idx_pitch < N) return fail(SSQB_EINVAL, "idx_pitch smaller than N");
  }
  if (gxr && !icwt_weights) return fail(SSQB_EINVAL, "gxr needs icwt_weights");
  return SSQB_OK;
}

size_t ssqb_cwt_adjoint_workspace_bytes(int B, int Npad, int na, int precision) {
  if (B < 1 || na < 1 || !is_pow2(Npad) || !valid_precision(precision)) return 0;
  return cwt_adjoint_workspace(B, Npad, na, data_prec(precision) == SSQB_F64);
}

int ssqb_cwt_adjoint(const void* gWx, const void* gTx, const uint16_t* idx, int idx_pitch,
                     const double* sq_weights, int nbins, const void* gxr,
                     const double* icwt_weights, int B, int N, int Npad, int n1, int padtype,
                     const double* scales, int na, const ssqb_wavelet* wavelet, int precision,
                     void* gx, int accumulate, void* workspace, size_t workspace_bytes,
                     void* stream) {
  if (!scales || !gx || !workspace) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || N < 1 || na < 1) return fail(SSQB_EINVAL, "B, N and na must be >= 1");
  if (B > 65535 || na > 65535) return fail(SSQB_EINVAL, "B and na must be <= 65535");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  if (!is_pow2(Npad) || Npad < 8 || Npad > (1 << 22))
    return fail(SSQB_EUNSUPPORTED, "Npad must be a power of two in [8, 2^22]");
  if (Npad < N || n1 < 0 || n1 + N > Npad) return fail(SSQB_EINVAL, "bad padding geometry");
  if (padtype < 0 || padtype > 5) return fail(SSQB_EINVAL, "unknown padtype");
  if (padtype == 3)
    return fail(SSQB_EUNSUPPORTED, "the adjoint of replicate padding is not implemented");
  if (idx_pitch == 0) idx_pitch = N;
  int r = check_adj_sources(gWx, gTx, idx, idx_pitch, sq_weights, nbins, gxr, icwt_weights, N);
  if (r) return r;
  WavDev wd;
  r = check_wavelet(wavelet, &wd);
  if (r) return r;
  const bool f64 = data_prec(precision) == SSQB_F64;
  const size_t need = cwt_adjoint_workspace(B, Npad, 1, f64);
  if (workspace_bytes < need)
    return fail(SSQB_EWORKSPACE, "workspace too small: need " + std::to_string(need) +
                                     " bytes");
  Tables tb;
  r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  int e;
  if (f64) {
    AdjSources<double2> src{(const double2*)gWx, (const double2*)gTx, idx, idx_pitch, nbins,
                            sq_weights, (const double*)gxr, icwt_weights};
    e = run_cwt_adjoint_f64(src, B, N, Npad, n1, padtype, scales, na, wd, (double*)gx,
                            accumulate, workspace, workspace_bytes, tb, st);
  } else {
    AdjSources<float2> src{(const float2*)gWx, (const float2*)gTx, idx, idx_pitch, nbins,
                           sq_weights, (const float*)gxr, icwt_weights};
    e = run_cwt_adjoint_f32(src, B, N, Npad, n1, padtype, scales, na, wd, (float*)gx,
                            accumulate, workspace, workspace_bytes, tb, st);
  }
  if (e) return cuda_fail((cudaError_t)e, "cwt adjoint launch");
  return SSQB_OK;
}

size_t ssqb_stft_adjoint_workspace_bytes(int B, int N, int n_fft, int hop, int precision) {
  if (B < 1 || N < 1 || hop < 1 || n_fft < 1 || !valid_precision(precision)) return 0;
  const size_t rs = data_prec(precision) == SSQB_F64 ? sizeof(double) : sizeof(float);
  return (size_t)B * n_fft * ((size_t)(N - 1) / hop + 1) * rs;
}

int ssqb_stft_adjoint(const void* gSx, const void* gTx, const uint16_t* idx, int idx_pitch,
                      const double* sq_weights, int B, int N, int n_fft, int hop, int n1,
                      int padtype, int modulated, const double* window, int precision,
                      void* gx, int accumulate, void* workspace, size_t workspace_bytes,
                      void* stream) {
  if (!window || !gx || !workspace) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || N < 1 || hop < 1) return fail(SSQB_EINVAL, "B, N and hop must be >= 1");
  if (B > 65535) return fail(SSQB_EINVAL, "B must be <= 65535");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  const bool pow2 = is_pow2(n_fft);
  int log2M = 0;
  while ((1 << log2M) < 2 * n_fft - 1) ++log2M;
  if (pow2 ? (n_fft < 8 || n_fft > 4096)
           : (n_fft < 4 || (1 << log2M) > FftCfg<double2>::TILE))
    return fail(SSQB_EUNSUPPORTED,
                "n_fft must be a power of two in [8, 4096] or any length in [4, " +
                    std::to_string((FftCfg<double2>::TILE + 1) / 2) + "]");
  const bool f64 = data_prec(precision) == SSQB_F64;
  if (pow2 && f64 && n_fft > FftCfg<double2>::TILE)
    return fail(SSQB_EUNSUPPORTED, "n_fft above " + std::to_string(FftCfg<double2>::TILE) +
                                       " needs float32 data");
  if (padtype < 0 || padtype > 5) return fail(SSQB_EINVAL, "unknown padtype");
  if (padtype == 3)
    return fail(SSQB_EUNSUPPORTED, "the adjoint of replicate padding is not implemented");
  if (n1 < 0 || n1 > n_fft) return fail(SSQB_EINVAL, "bad padding geometry");
  const int nframes = (N - 1) / hop + 1;
  if (idx_pitch == 0) idx_pitch = nframes;
  const int nrow = n_fft / 2 + 1;
  int r = check_adj_sources(gSx, gTx, idx, idx_pitch, sq_weights, nrow, nullptr, nullptr,
                            nframes);
  if (r) return r;
  const size_t need = ssqb_stft_adjoint_workspace_bytes(B, N, n_fft, hop, precision);
  if (workspace_bytes < need)
    return fail(SSQB_EWORKSPACE, "workspace too small: need " + std::to_string(need) +
                                     " bytes");
  Tables tb;
  r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  int e;
  if (f64) {
    AdjSources<double2> src{(const double2*)gSx, (const double2*)gTx, idx, idx_pitch, nrow,
                            sq_weights, nullptr, nullptr};
    e = run_stft_adjoint_f64(src, B, N, n_fft, hop, n1, padtype, modulated ? 1 : 0, window,
                             (double*)gx, accumulate, workspace, tb, st);
  } else {
    AdjSources<float2> src{(const float2*)gSx, (const float2*)gTx, idx, idx_pitch, nrow,
                           sq_weights, nullptr, nullptr};
    e = run_stft_adjoint_f32(src, B, N, n_fft, hop, n1, padtype, modulated ? 1 : 0, window,
                             (float*)gx, accumulate, workspace, tb, st);
  }
  if (e) return cuda_fail((cudaError_t)e, "stft adjoint launch");
  return SSQB_OK;
}

int ssqb_phase_diff(const void* Wx, int B, int na, int ncol, int col0, int M, int mode,
                    int difforder, double dt, double gamma, int precision, void* w,
                    void* stream) {
  if (!Wx || !w) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || na < 1 || M < 2) return fail(SSQB_EINVAL, "B, na must be >= 1 and M >= 2");
  if (col0 < 0 || ncol < 1 || (long long)col0 + M > ncol)
    return fail(SSQB_EINVAL, "columns col0 .. col0+M-1 must lie in the row");
  if (mode != 1 && mode != 2) return fail(SSQB_EINVAL, "mode must be 1 (phase) or 2 (numeric)");
  if (mode == 2 && difforder != 1 && difforder != 2 && difforder != 4)
    return fail(SSQB_EINVAL, "difforder must be 1, 2 or 4");
  if (mode == 2 && !(dt > 0)) return fail(SSQB_EINVAL, "dt must be > 0");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  const long long rows = (long long)B * na;
  if (rows > 0x7fffffffLL) return fail(SSQB_EINVAL, "too many rows");
  cudaStream_t st = (cudaStream_t)stream;
  int e;
  if (data_prec(precision) == SSQB_F64)
    e = run_phase_diff_f64((const double2*)Wx, rows, ncol, col0, M, mode, difforder, dt, gamma,
                           (double*)w, st);
  else
    e = run_phase_diff_f32((const float2*)Wx, rows, ncol, col0, M, mode, difforder, dt, gamma,
                           (float*)w, st);
  if (e) return cuda_fail((cudaError_t)e, "phase_diff launch");
  return SSQB_OK;
}

static size_t trigdiff_chunk(int rows, int Npad) {
  const size_t per = (size_t)Npad * sizeof(double2);
  size_t c = ((size_t)256 << 20) / per;
  if (c < 1) c = 1;
  return c < (size_t)rows ? c : (size_t)rows;
}

size_t ssqb_trigdiff_workspace_bytes(int rows, int Npad) {
  if (rows < 1 || !is_pow2(Npad)) return 0;
  const size_t z = kZBudgetBytes > (size_t)Npad * sizeof(double2)
                       ? kZBudgetBytes : (size_t)Npad * sizeof(double2);
  return trigdiff_chunk(rows, Npad) * Npad * sizeof(double2) + z;
}

int ssqb_trigdiff(const void* A, int rows, int M, int Npad, int n1, int padtype, double fs,
                  int out_off, int N_out, int precision, void* out, void* workspace,
                  size_t workspace_bytes, void* stream) {
  if (!A || !out || !workspace) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (rows < 1 || M < 1 || N_out < 1) return fail(SSQB_EINVAL, "rows, M, N_out must be >= 1");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  if (!is_pow2(Npad) || Npad < 8 || Npad > (1 << 22))
    return fail(SSQB_EUNSUPPORTED, "Npad must be a power of two in [8, 2^22]");
  if (padtype < 0 || padtype > 5) return fail(SSQB_EINVAL, "unknown padtype");
  if (n1 < 0 || (long long)n1 + M > Npad) return fail(SSQB_EINVAL, "bad padding geometry");
  if (padtype == 5 && (n1 != 0 || M != Npad))
    return fail(SSQB_EINVAL, "padtype 5 (none) needs M == Npad and n1 == 0");
  if (out_off < 0 || (long long)out_off + N_out > Npad)
    return fail(SSQB_EINVAL, "output columns must lie in [0, Npad)");
  const size_t need = ssqb_trigdiff_workspace_bytes(rows, Npad);
  if (workspace_bytes < need)
    return fail(SSQB_EWORKSPACE, "workspace too small: need " + std::to_string(need) +
                                     " bytes");
  Tables tb;
  int r = get_tables(&tb);
  if (r) return r;
  const int chunk = (int)trigdiff_chunk(rows, Npad);
  double2* xh = (double2*)workspace;
  double2* Z = xh + (size_t)chunk * Npad;
  const size_t zcap = (workspace_bytes - (size_t)chunk * Npad * sizeof(double2)) /
                      sizeof(double2);
  const int e = run_trigdiff(A, data_prec(precision) == SSQB_F64, rows, M, Npad, n1, padtype,
                             fs, out_off, N_out, out, xh, chunk, Z, zcap, tb,
                             (cudaStream_t)stream);
  if (e) return cuda_fail((cudaError_t)e, "trigdiff launch");
  return SSQB_OK;
}

size_t ssqb_istft_workspace_bytes(int B, int n_fft, int n_frames, int precision) {
  if (B < 1 || n_frames < 1 || n_fft < 1 || !valid_precision(precision)) return 0;
  const size_t rs = data_prec(precision) == SSQB_F64 ? sizeof(double) : sizeof(float);
  return (size_t)B * n_fft * (size_t)n_frames * rs;
}

int ssqb_istft(const void* Sx, int B, int n_fft, int n_frames, int hop, int N, int modulated,
               const double* wa, const double* w1, double tiny, int precision, void* x,
               void* workspace, size_t workspace_bytes, void* stream) {
  if (!Sx || !wa || !w1 || !x || !workspace) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || N < 1 || hop < 1 || n_frames < 1)
    return fail(SSQB_EINVAL, "B, N, hop and n_frames must be >= 1");
  if (B > 65535) return fail(SSQB_EINVAL, "B must be <= 65535");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  const bool pow2 = is_pow2(n_fft);
  int log2M = 0;
  while ((1 << log2M) < 2 * n_fft - 1) ++log2M;
  if (pow2 ? (n_fft < 8 || n_fft > 4096)
           : (n_fft < 4 || (1 << log2M) > FftCfg<double2>::TILE))
    return fail(SSQB_EUNSUPPORTED,
                "n_fft must be a power of two in [8, 4096] or any length in [4, " +
                    std::to_string((FftCfg<double2>::TILE + 1) / 2) + "]");
  const bool f64 = data_prec(precision) == SSQB_F64;
  if (pow2 && f64 && n_fft > FftCfg<double2>::TILE)
    return fail(SSQB_EUNSUPPORTED, "n_fft above " + std::to_string(FftCfg<double2>::TILE) +
                                       " needs float32 data");
  if ((long long)(n_frames - 1) * hop > (long long)N - 1)
    return fail(SSQB_EINVAL, "frames end past the signal: need (n_frames - 1) * hop <= N - 1");
  if (!(tiny >= 0)) return fail(SSQB_EINVAL, "tiny must be >= 0");
  const size_t need = ssqb_istft_workspace_bytes(B, n_fft, n_frames, precision);
  if (workspace_bytes < need)
    return fail(SSQB_EWORKSPACE, "workspace too small: need " + std::to_string(need) +
                                     " bytes");
  Tables tb;
  int r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  int e;
  if (f64)
    e = run_istft_f64((const double2*)Sx, B, N, n_fft, hop, n_frames, modulated ? 1 : 0, wa,
                      w1, tiny, (double*)x, workspace, tb, st);
  else
    e = run_istft_f32((const float2*)Sx, B, N, n_fft, hop, n_frames, modulated ? 1 : 0, wa,
                      w1, tiny, (float*)x, workspace, tb, st);
  if (e) return cuda_fail((cudaError_t)e, "istft launch");
  return SSQB_OK;
}

static int wx_adjoint(const void* gTx, const uint16_t* idx, int idx_pitch,
                      const double* sq_weights, int nbins, const void* gxr,
                      const double* icwt_weights, int B, int na, int N, int precision,
                      void* gWx, int accumulate, void* stream) {
  if (!gWx) return fail(SSQB_EINVAL, "NULL pointer argument");
  if (B < 1 || N < 1 || na < 1) return fail(SSQB_EINVAL, "B, N and na must be >= 1");
  if (B > 65535 || na > 65535) return fail(SSQB_EINVAL, "B and na must be <= 65535");
  if (!valid_precision(precision))
    return fail(SSQB_EINVAL, "precision must be SSQB_F32, SSQB_F64 or SSQB_F32X");
  if (idx_pitch == 0) idx_pitch = N;
  int r = check_adj_sources(nullptr, gTx, idx, idx_pitch, sq_weights, nbins, gxr,
                            icwt_weights, N);
  if (r) return r;
  Tables tb;
  r = get_tables(&tb);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  int e;
  if (data_prec(precision) == SSQB_F64) {
    AdjSources<double2> src{nullptr, (const double2*)gTx, idx, idx_pitch, nbins, sq_weights,
                            (const double*)gxr, icwt_weights};
    e = run_wx_adjoint_f64(src, B, na, N, (double2*)gWx, accumulate, tb.status, st);
  } else {
    AdjSources<float2> src{nullptr, (const float2*)gTx, idx, idx_pitch, nbins, sq_weights,
                           (const float*)gxr, icwt_weights};
    e = run_wx_adjoint_f32(src, B, na, N, (float2*)gWx, accumulate, tb.status, st);
  }
  if (e) return cuda_fail((cudaError_t)e, "adjoint launch");
  return SSQB_OK;
}

int ssqb_squeeze_adjoint(const void* gTx, const uint16_t* idx, int idx_pitch,
                         const double* row_weights, int B, int na, int N, int nbins,
                         int precision, void* gWx, int accumulate, void* stream) {
  if (!gTx) return fail(SSQB_EINVAL, "NULL pointer argument");
  return wx_adjoint(gTx, idx, idx_pitch, row_weights, nbins, nullptr, nullptr, B, na, N,
                    precision, gWx, accumulate, stream);
}

int ssqb_icwt_adjoint(const void* gx, const double* row_weights, int B, int na, int N,
                      int precision, void* gWx, int accumulate, void* stream) {
  if (!gx) return fail(SSQB_EINVAL, "NULL pointer argument");
  return wx_adjoint(nullptr, nullptr, 0, nullptr, 0, gx, row_weights, B, na, N, precision,
                    gWx, accumulate, stream);
}

}  // extern "C"
