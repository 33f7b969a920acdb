// Tile-FFT kernel instantiations for x_hat and the fused CWT, and their
// host launchers (one pass when Npad fits a tile, else two passes).
#include "tile_launch.cuh"

namespace ssqb {

// When set, launchers count their launches here instead of launching.
static thread_local int* t_count = nullptr;
void set_launch_counter(int* c) { t_count = c; }
int* launch_counter() { return t_count; }

static thread_local bool t_aux_off = false;
void set_aux_streams(bool on) { t_aux_off = !on; }

AuxStream* aux_stream() {
  if (t_aux_off) return nullptr;
  static thread_local AuxStream t_aux[256];
  static thread_local bool t_made[256], t_bad[256];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return nullptr;
  if (t_bad[dev]) return nullptr;
  if (!t_made[dev]) {
    AuxStream a{};
    if (cudaStreamCreateWithFlags(&a.s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&a.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&a.join, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      t_bad[dev] = true;
      return nullptr;
    }
    t_aux[dev] = a;
    t_made[dev] = true;
  }
  return &t_aux[dev];
}

int run_xhat_f32(const float* x, int B, int N, int Npad, int n1, int padtype,
                 double2* xh, double2* Z, size_t zcap, const Tables& tb, cudaStream_t st) {
  XhatOp<float> op{x, xh, N, Npad, n1, padtype};
  return run_tile<XhatOp<float>, double2, -1>(op, B, 1, ilog2(Npad), Z, zcap, tb, st);
}

int run_xhat_f64(const double* x, int B, int N, int Npad, int n1, int padtype,
                 double2* xh, double2* Z, size_t zcap, const Tables& tb, cudaStream_t st) {
  XhatOp<double> op{x, xh, N, Npad, n1, padtype};
  return run_tile<XhatOp<double>, double2, -1>(op, B, 1, ilog2(Npad), Z, zcap, tb, st);
}

// tile passes for rows [0, two_pass_rows), then each band group
template <class Op, typename C>
static int run_cwt_t(const Op& op, int B, int log2L, C* Z, size_t zcap, const Tables& tb,
                     cudaStream_t st, const BandPlan* bp) {
  if (!bp || bp->ngroups == 0 || !two_pass<C>(log2L))
    return run_tile_signals<Op, C, 1>(op, B, op.na, log2L, Z, zcap, tb, st);
  if (bp->two_pass_rows > 0) {
    Op o = op;
    o.nrun = bp->two_pass_rows;
    const int e = run_tile_signals<Op, C, 1>(o, B, o.nrun, log2L, Z, zcap, tb, st);
    if (e) return e;
  }
  for (int g = 0; g < bp->ngroups; ++g) {
    const int e = run_band<Op, C, 1>(op, B, log2L, bp->logM[g], Z, zcap, bp->r0[g],
                                     bp->nrows[g], tb, st);
    if (e) return e;
  }
  return 0;
}

int run_cwt_f32(const CwtOp<float2>& op, int B, int log2L, float2* Z, size_t zcap,
                const Tables& tb, cudaStream_t st, const BandPlan* bp) {
  return run_cwt_t(op, B, log2L, Z, zcap, tb, st, bp);
}

int run_cwt_f64(const CwtOp<double2>& op, int B, int log2L, double2* Z, size_t zcap,
                const Tables& tb, cudaStream_t st, const BandPlan* bp) {
  return run_cwt_t(op, B, log2L, Z, zcap, tb, st, bp);
}

int run_cwt_f32x(const CwtOp<double2, float2>& op, int B, int log2L, double2* Z,
                 size_t zcap, const Tables& tb, cudaStream_t st, const BandPlan* bp) {
  return run_cwt_t(op, B, log2L, Z, zcap, tb, st, bp);
}

// trigdiff: rows in chunks of `chunk` through the spectrum buffer xh
template <typename TC, typename OC>
static int run_trigdiff_t(const TC* A, int rows, int M, int Npad, int n1, int padtype,
                          double fs, int out_off, int N_out, OC* out, double2* xh, int chunk,
                          double2* Z, size_t zcap, const Tables& tb, cudaStream_t st) {
  const int m = ilog2(Npad);
  for (int r0 = 0; r0 < rows; r0 += chunk) {
    const int nr = (rows - r0) < chunk ? (rows - r0) : chunk;
    RowFftOp<TC> f{A, xh, M, Npad, n1, padtype, r0, nr};
    int e = run_tile<RowFftOp<TC>, double2, -1>(f, 1, nr, m, Z, zcap, tb, st);
    if (e) return e;
    RowDiffOp<OC> d{xh, out, Npad, r0, nr, out_off, N_out, 2.0 * M_PI / Npad * fs,
                    1.0 / Npad};
    e = run_tile<RowDiffOp<OC>, double2, 1>(d, 1, nr, m, Z, zcap, tb, st);
    if (e) return e;
  }
  return 0;
}

int run_trigdiff(const void* A, bool f64, int rows, int M, int Npad, int n1, int padtype,
                 double fs, int out_off, int N_out, void* out, double2* xh, int chunk,
                 double2* Z, size_t zcap, const Tables& tb, cudaStream_t st) {
  if (f64)
    return run_trigdiff_t<double2, double2>((const double2*)A, rows, M, Npad, n1, padtype, fs,
                                            out_off, N_out, (double2*)out, xh, chunk, Z, zcap,
                                            tb, st);
  return run_trigdiff_t<float2, float2>((const float2*)A, rows, M, Npad, n1, padtype, fs,
                                        out_off, N_out, (float2*)out, xh, chunk, Z, zcap, tb,
                                        st);
}

int run_xhat_batch_f32(const float* x, const SigDesc* desc, int nsig, int Npad, int padtype,
                       double2* xh, double2* Z, size_t zcap, const Tables& tb,
                       cudaStream_t st) {
  XhatBatchOp<float> op{x, xh, desc, Npad, padtype};
  return run_batch<XhatBatchOp<float>, double2, -1>(op, nsig, 1, ilog2(Npad), Z, zcap, tb,
                                                    st);
}

// rows [0, band_from) by the tile passes, [band_from, max_na) by the band pass
template <class BOp, typename C>
static int run_cwt_batch_t(const BOp& op, int nsig, int max_na, int log2L, int band_log,
                           C* Z, size_t zcap, const Tables& tb, cudaStream_t st) {
  BOp o = op;  // single-pass lengths and no band rows: every row by the tile passes
  if (!(op.band_from < max_na && two_pass<C>(log2L))) o.band_from = 0x7fffffff;
  const int bf = o.band_from < max_na ? o.band_from : max_na;
  if (bf > 0) {
    const int e = run_batch<BOp, C, 1>(o, nsig, bf, log2L, Z, zcap, tb, st);
    if (e) return e;
  }
  if (bf < max_na)
    return run_band<BOp, C, 1>(o, nsig, log2L, band_log, Z, zcap, bf, max_na - bf, tb, st);
  return 0;
}

int run_cwt_batch_f32x(const CwtBatchOp<double2, float2>& op, int nsig, int max_na,
                       int log2L, int band_log, double2* Z, size_t zcap, const Tables& tb,
                       cudaStream_t st) {
  return run_cwt_batch_t(op, nsig, max_na, log2L, band_log, Z, zcap, tb, st);
}

int run_cwt_batch_f32(const CwtBatchOp<float2, float2>& op, int nsig, int max_na, int log2L,
                      int band_log, float2* Z, size_t zcap, const Tables& tb,
                      cudaStream_t st) {
  return run_cwt_batch_t(op, nsig, max_na, log2L, band_log, Z, zcap, tb, st);
}

}  // namespace ssqb
