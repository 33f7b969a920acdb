// Host-side launchers shared between the kernel translation units and the
// C-ABI layer. Each returns 0 or a cudaError_t value.
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include "ssqb_ops.cuh"

namespace ssqb {

// row tile of the two-pass transform: as many rows as the intermediate
// holds (zcap complex elements, at least one row), then trimmed so that the
// CTA count of a launch fills whole waves of `slots` resident CTAs
inline int rows_per_tile(size_t zcap_elems, int B, int narr, int log2L, int nrows,
                         int ctas_per_row = 0, int slots = 0) {
  const size_t per = (size_t)B * narr * ((size_t)1 << log2L);
  size_t s = per ? zcap_elems / per : 0;
  if (s < 1) s = 1;
  if (s > (size_t)nrows) s = nrows;
  if (s > 65535) s = 65535;
  if (ctas_per_row > 0 && slots > 0 && s > 1) {
    double best = 2.0;
    size_t pick = s;
    for (size_t r = s; r >= (s + 1) / 2 && r >= 1; --r) {
      const double c = (double)r * ctas_per_row * B;
      const double waves = c / slots;
      const double waste = (std::ceil(waves) - waves) / std::ceil(waves);
      if (waste < best - 0.02) { best = waste; pick = r; }
      if (r == 1) break;
    }
    s = pick;
  }
  return (int)s;
}

// Budget of the two-pass intermediate of one ssqb_cwt call, bytes. 64 MB
// keeps it within the 126 MB L2 together with the spectrum and the streaming
// outputs. Longer transforms measured faster with larger row tiles, the
// intermediate then partly in DRAM (cwt ms, same call): at N = 160,000
// (Npad 2^18) 64 MB 1.878, 256 MB 1.832, 512 MB 1.773; at 2^20 18.97, 18.74,
// 18.57; at N = 40,000 (Npad 2^16) 0.472 -> 0.459 with 256 MB. At N = 10,000
// (2^14) a large budget puts every row in one tile and the two streams stop
// overlapping (0.139 -> 0.155 ms), so short transforms keep 64 MB.
#ifndef SSQB_Z_MB
#define SSQB_Z_MB 64
#endif
constexpr size_t kZBudgetBytes = (size_t)SSQB_Z_MB << 20;
inline size_t cwt_z_budget(int log2L) {
  if (log2L >= 17) return (size_t)512 << 20;
  if (log2L == 16) return (size_t)256 << 20;
  return kZBudgetBytes;
}

// Row tiles of one transform alternate between the caller's stream and an
// auxiliary stream of this host thread (fork and join through events), each
// with its own half of the intermediate, so that one tile's last wave
// overlaps the next tile's first.
#ifndef SSQB_DUAL_STREAM
#define SSQB_DUAL_STREAM 1
#endif
struct AuxStream {
  cudaStream_t s;
  cudaEvent_t fork, join;
};
AuxStream* aux_stream();  // NULL if it cannot be created or is switched off
void set_aux_streams(bool on);  // this host thread; on by default

// single pass when L fits one tile (4096 float2 / 2048 double2 elements);
// else two passes with log2(L2) = m/2
template <typename C> inline bool two_pass(int log2L) {
  return (1 << log2L) > FftCfg<C>::TILE;
}

int run_xhat_f32(const float* x, int B, int N, int Npad, int n1, int padtype,
                 double2* xh, double2* Z, size_t zcap, const Tables& tb,
                 cudaStream_t st);
int run_xhat_f64(const double* x, int B, int N, int Npad, int n1, int padtype,
                 double2* xh, double2* Z, size_t zcap, const Tables& tb,
                 cudaStream_t st);
// Rows of a CWT call whose wavelet band fits M = 2^logM bins (a suffix of
// the rows, in groups of one M each) take the band-limited single pass; rows
// [0, two_pass_rows) take the tile passes. Built on the host from the scale
// values (cwt_band_plan); without it every row takes the tile passes.
struct BandPlan {
  static constexpr int kMaxGroups = 16;
  int two_pass_rows;
  int ngroups;
  int r0[kMaxGroups], nrows[kMaxGroups], logM[kMaxGroups];
};
int run_cwt_f32(const CwtOp<float2>& op, int B, int log2L, float2* Z, size_t zcap,
                const Tables& tb, cudaStream_t st, const BandPlan* bp = nullptr);
int run_cwt_f64(const CwtOp<double2>& op, int B, int log2L, double2* Z, size_t zcap,
                const Tables& tb, cudaStream_t st, const BandPlan* bp = nullptr);
int run_cwt_f32x(const CwtOp<double2, float2>& op, int B, int log2L, double2* Z,
                 size_t zcap, const Tables& tb, cudaStream_t st,
                 const BandPlan* bp = nullptr);
int run_istft_frames_any_f32(const float2* Sx, int B, int L, int nframes, float* gu,
                             const Tables& tb, cudaStream_t st);
int run_istft_frames_any_f64(const double2* Sx, int B, int L, int nframes, double* gu,
                             const Tables& tb, cudaStream_t st);
int run_adj_frames_any_f32(const AdjSources<float2>& src, int B, int L, int nframes,
                           float* gu, const Tables& tb, cudaStream_t st);
int run_adj_frames_any_f64(const AdjSources<double2>& src, int B, int L, int nframes,
                           double* gu, const Tables& tb, cudaStream_t st);
int run_stft_any_f32x(const StftOp<float, double2, float2>& op, int B, int log2M,
                      const Tables& tb, cudaStream_t st);
int run_stft_any_f64(const StftOp<double, double2>& op, int B, int log2M, const Tables& tb,
                     cudaStream_t st);
int run_stft_f32(const StftOp<float, float2>& op, int B, int log2L,
                 const Tables& tb, cudaStream_t st);
int run_stft_f64(const StftOp<double, double2>& op, int B, int log2L,
                 const Tables& tb, cudaStream_t st);
int run_stft_f32x(const StftOp<float, double2, float2>& op, int B, int log2L,
                  const Tables& tb, cudaStream_t st);

// squeeze; src_kind 0 = uint16 index (rows of idx_pitch), 1 = phase from dWx
// (cwt or stft), 2 = w
int run_squeeze_f32(const float2* Wx, int src_kind, const void* src, int idx_pitch,
                    const double* sfs, const BinDev& bins, double gamma, const double* cst,
                    int B, int na, int N, int nbins, float2* Tx, int* status,
                    cudaStream_t st);
int run_squeeze_f64(const double2* Wx, int src_kind, const void* src, int idx_pitch,
                    const double* sfs, const BinDev& bins, double gamma, const double* cst,
                    int B, int na, int N, int nbins, double2* Tx, int* status,
                    cudaStream_t st);

int run_icwt(const void* Wx, const double* w, const double* x_mean, double mean_weight,
             int B, int na, int N, int precision, void* x, cudaStream_t st);
int run_issq(const void* Tx, int nrows, int N, const int* cc, const int* cw, int K,
             double scale, int precision, void* x, cudaStream_t st);

// count launches of this host thread into *c instead of launching (NULL:
// launch again)
void set_launch_counter(int* c);
int* launch_counter();

// batches of uneven lengths sharing one padded length (float32 data)
int run_trigdiff(const void* A, bool f64, int rows, int M, int Npad, int n1, int padtype,
                 double fs, int out_off, int N_out, void* out, double2* xh, int chunk,
                 double2* Z, size_t zcap, const Tables& tb, cudaStream_t st);
int run_xhat_batch_f32(const float* x, const SigDesc* desc, int nsig, int Npad, int padtype,
                       double2* xh, double2* Z, size_t zcap, const Tables& tb,
                       cudaStream_t st);
// op.band_from < max_na: rows from there take the band pass at 2^band_log bins
int run_cwt_batch_f32x(const CwtBatchOp<double2, float2>& op, int nsig, int max_na,
                       int log2L, int band_log, double2* Z, size_t zcap, const Tables& tb,
                       cudaStream_t st);
int run_cwt_batch_f32(const CwtBatchOp<float2, float2>& op, int nsig, int max_na, int log2L,
                      int band_log, float2* Z, size_t zcap, const Tables& tb,
                      cudaStream_t st);
int run_squeeze_batch_f32(const float2* Wx, const uint16_t* idx, const SigDesc* desc,
                          int nsig, int max_na, int max_N, float2* Tx, int* status,
                          cudaStream_t st);

// ridge extraction (k_ridges.cu)
size_t ridges_workspace(int nf, int N, bool f64);
int run_ridges(const void* Tf, int nf, int N, const void* s, const void* scales, double penalty,
               int n_ridges, int bw, double eps, bool f64, int* idx_out, void* f_out,
               void* e_out, void* ws, cudaStream_t st);

// adjoints (reverse-mode differentiation)
constexpr size_t kAdjChunkBytes = (size_t)64 << 20;  // row chunk: Y + Z
size_t cwt_adjoint_workspace(int B, int Npad, int na, bool f64);
int run_cwt_adjoint_f32(const AdjSources<float2>& src, int B, int N, int Npad, int n1,
                        int padtype, const double* scales, int na, const WavDev& wd, float* gx,
                        int accumulate, void* ws, size_t ws_bytes, const Tables& tb,
                        cudaStream_t st);
int run_cwt_adjoint_f64(const AdjSources<double2>& src, int B, int N, int Npad, int n1,
                        int padtype, const double* scales, int na, const WavDev& wd,
                        double* gx, int accumulate, void* ws, size_t ws_bytes,
                        const Tables& tb, cudaStream_t st);
int run_stft_adjoint_f32(const AdjSources<float2>& src, int B, int N, int L, int hop, int n1,
                         int padtype, int modulated, const double* win, float* gx,
                         int accumulate, void* ws, const Tables& tb, cudaStream_t st);
int run_stft_adjoint_f64(const AdjSources<double2>& src, int B, int N, int L, int hop, int n1,
                         int padtype, int modulated, const double* win, double* gx,
                         int accumulate, void* ws, const Tables& tb, cudaStream_t st);
int run_istft_f32(const float2* Sx, int B, int N, int L, int hop, int nframes, int modulated,
                  const double* wa, const double* w1, double tiny, float* x, void* ws,
                  const Tables& tb, cudaStream_t st);
int run_istft_f64(const double2* Sx, int B, int N, int L, int hop, int nframes, int modulated,
                  const double* wa, const double* w1, double tiny, double* x, void* ws,
                  const Tables& tb, cudaStream_t st);
int run_phase_diff_f32(const float2* Wx, long long rows, int ncol, int col0, int M, int mode,
                       int order, double dt, double gamma, float* w, cudaStream_t st);
int run_phase_diff_f64(const double2* Wx, long long rows, int ncol, int col0, int M, int mode,
                       int order, double dt, double gamma, double* w, cudaStream_t st);
int run_wx_adjoint_f32(const AdjSources<float2>& src, int B, int na, int N, float2* gWx,
                       int accumulate, int* status, cudaStream_t st);
int run_wx_adjoint_f64(const AdjSources<double2>& src, int B, int na, int N, double2* gWx,
                       int accumulate, int* status, cudaStream_t st);

}  // namespace ssqb
