/* ssqb: B200-native (sm_100a) synchrosqueezing hot path, C ABI.
 *
 * Every entry point takes device pointers, sizes and a CUDA stream
 * (`stream`, a cudaStream_t passed as void*, NULL = legacy default stream),
 * returns an int status (SSQB_OK = 0) and allocates nothing: outputs and
 * workspaces belong to the caller. Work is enqueued on `stream`; calls return
 * before it completes. Layouts are C-contiguous; complex arrays are
 * interleaved (re, im) pairs of float (SSQB_F32) or double (SSQB_F64).
 *
 * Shapes: B signals of N samples each; na rows (CWT scales or STFT
 * frequencies); nbins rows of Tx (= na for the transforms here).
 *
 * The entry points replace the GPU seams of ssqueezepy (paths are relative
 * to its source tree):
 *   ssqb_cwt            _cwt.py:250-311 (pad, fft, Psih*xh, two ifft,
 *                       unpad) + algos.py:743-781 (phase_cwt_gpu) fused,
 *                       and the bin search of algos.py:1008-1128
 *   ssqb_squeeze        utils/gpu_utils.py:10-14 launching the
 *                       `ssq_cwt_*` / `ssq_stft` kernels of
 *                       algos.py:1007-1167 (here reading a bin index)
 *   ssqb_ssqueeze_fast  algos.py:126-150 (ssqueeze_fast) on the GPU
 *   ssqb_indexed_sum    algos.py:153-169 (indexed_sum_onfly) on the GPU
 *   ssqb_stft           _stft.py:127-181 + utils/stft_utils.py:101-138
 *                       (buffer) + algos.py:818-856 (phase_stft_gpu) fused
 */
#ifndef SSQB_H_
#define SSQB_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SSQB_API __attribute__((visibility("default")))
#else
#define SSQB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SSQB_OK = 0,
  SSQB_EINVAL = 1,        /* bad argument (message in ssqb_last_error) */
  SSQB_EUNSUPPORTED = 2,  /* valid but not supported (e.g. non power-of-2 length) */
  SSQB_ECUDA = 3,         /* CUDA runtime error */
  SSQB_EWORKSPACE = 4     /* workspace smaller than required */
};

/* precision: SSQB_F32 float32 data and arithmetic; SSQB_F64 float64 data
 * and arithmetic; SSQB_F32X float32 data (x, Wx, Sx, Tx, w) with float64
 * arithmetic inside the transforms, so bin decisions match the float64 path
 * except at exact ties. */
enum { SSQB_F32 = 0, SSQB_F64 = 1, SSQB_F32X = 2 };

/* padtype: 0 zero, 1 reflect, 2 symmetric, 3 replicate, 4 wrap
 * (utils/common.py:54-158) */

/* Frequency-domain wavelet (wavelets.py:498-530, _gmw.py:187-251).
 * kind 0 Morlet:   p = {mu, ks = exp(-mu^2/2), C1 = sqrt(2) cs pi^(1/4), 0}
 * kind 1 GMW L1:   p = {gamma, beta, wc = (beta/gamma)^(1/gamma), log(wc)}
 * kind 2 GMW L2:   p = {gamma, beta, wc, sqrt(2 pi gamma 2^r / Gamma(r))}
 * band = {w_lo, w_hi}: psih is taken as 0 outside [w_lo, w_hi] (where it is
 * below ~1e-30 of its peak); band[0] >= band[1] evaluates everywhere.
 * npoly > 0 (GMW only; at most 8): higher-order GMW (_gmw.py:268-347). The
 * constant factor (2 for L1, p[3] for L2) becomes the polynomial
 * C(w) = sum_{m < npoly} kc[m] (2 w^gamma)^m, Laguerre constants times the
 * order-k norm (_gmw.py:368-396); an average over orders (_cwt.py:517-610)
 * is the mean of the orders' coefficient vectors. */
typedef struct ssqb_wavelet {
  int32_t kind;
  int32_t npoly;
  double p[4];
  double band[2];
  double kc[8];
} ssqb_wavelet;

/* Bin mapping of the squeeze (algos.py:81-87, 356-374).
 * mode 0 log:           p = {vlmin, dvl}
 * mode 1 log-piecewise: p = {vlmin0, vlmin1, dvl0, dvl1}, idx1
 * mode 2 linear:        p = {vmin, dv}
 * flipud: k -> nbins-1-k (ssqueezing.py:13-15, algos.py:95) */
typedef struct ssqb_bins {
  int32_t mode;
  int32_t idx1;
  int32_t flipud;
  int32_t nbins;
  double p[4];
} ssqb_bins;

SSQB_API int ssqb_version(void);

/* Message of the last failing call on this host thread. */
SSQB_API const char* ssqb_last_error(void);

/* Copy and clear the device status word of the current device (0 = ok,
 * 1 = bin index out of range, 2 = padded index out of range, 3 = a bounded
 * wait on an asynchronous copy expired); synchronizes `stream`. */
SSQB_API int ssqb_device_status(void* stream, int* status_out);

/* Workspace bytes for ssqb_cwt: the float64 padded-signal spectrum plus
 * the two-pass intermediate for two tiles of rows: a 64 MB budget (kept in
 * L2) up to Npad = 32,768, 256 MB at 65,536 and 512 MB from 131,072 on
 * (larger row tiles measured faster there). Smaller workspaces down to the
 * minimum work too, with smaller row tiles. */
SSQB_API size_t ssqb_cwt_workspace_bytes(int B, int N, int Npad, int na, int precision);

/* Number of kernel launches one ssqb_cwt call makes with this workspace
 * size (padded-signal FFT plus CWT passes); no reference counterpart. */
SSQB_API int ssqb_cwt_launches(int B, int Npad, int na, int precision,
                               size_t workspace_bytes);

/* Fused CWT (replaces _cwt.py:250-311 with derivative=True, l1_norm=True,
 * plus the phase transform and bin search of algos.py:859-953):
 *   x      (B, N) float (F32) or double (F64)
 *   scales (na) double, device
 *   Wx     (B, na, N) complex, required; dWx optional (NULL)
 *   w      (B, na, N) real phase transform, optional (inf where |Wx|<gamma)
 *   idx    (B, na, idx_pitch) uint16 bin of each entry, 0xFFFF where
 *          |Wx|<=gamma; optional (needs `bins`); idx_pitch >= N columns (0 = N)
 * Npad is the padded length (a power of two, 8 <= Npad <= 2^22) and n1 the
 * left pad; dt = 1/fs. rpadded != 0 writes all Npad columns (outputs
 * (B, na, Npad), _cwt.py:293-306 with rpadded=True). */
SSQB_API int ssqb_cwt(const void* x, int B, int N, int Npad, int n1, int padtype, int rpadded,
             const double* scales, int na, const ssqb_wavelet* wavelet, double dt,
             const ssqb_bins* bins, double gamma, int precision,
             void* Wx, void* dWx, void* w, uint16_t* idx, int idx_pitch,
             void* workspace, size_t workspace_bytes, void* stream);

/* ssqb_cwt with the scale values also given on the host (`scales_host`, na
 * doubles equal to the device `scales`; NULL makes it ssqb_cwt). They let
 * the call plan per row: rows whose wavelet band spans at most half a
 * transform tile for Npad <= 65536, a quarter above (1024 / 512 bins with
 * float64 arithmetic, 2048 / 1024 with SSQB_F32), go through a band-limited
 * single pass (D = Npad / M transforms of the
 * twiddled band, M the band's power-of-two length, no two-pass
 * intermediate) instead of the four-step of the full padded length. Same
 * outputs, workspace and stream semantics as ssqb_cwt. No reference
 * counterpart (the reference multiplies the full padded spectrum and takes
 * full-length inverse FFTs of every row, _cwt.py:167-177). */
SSQB_API int ssqb_cwt_ex(const void* x, int B, int N, int Npad, int n1, int padtype,
                         int rpadded, const double* scales, const double* scales_host,
                         int na, const ssqb_wavelet* wavelet, double dt,
                         const ssqb_bins* bins, double gamma, int precision, void* Wx,
                         void* dWx, void* w, uint16_t* idx, int idx_pitch, void* workspace,
                         size_t workspace_bytes, void* stream);

/* Number of kernel launches one ssqb_cwt_ex call makes with these host
 * scales and this workspace size; no reference counterpart. */
SSQB_API int ssqb_cwt_ex_launches(int B, int Npad, int na, int precision,
                                  size_t workspace_bytes, const double* scales_host,
                                  const ssqb_wavelet* wavelet);

/* Squeeze from a bin index: Tx[b, idx, j] += Wx[b, i, j] * row_weights[i]
 * over i ascending (algos.py:859-984 accumulation order). idx rows have
 * idx_pitch columns (0 = N). Tx (B, nbins, N) is overwritten. */
SSQB_API int ssqb_squeeze(const void* Wx, const uint16_t* idx, int idx_pitch,
                          const double* row_weights, int B, int na, int N, int nbins,
                          int precision, void* Tx, void* stream);

/* Squeeze computing the phase transform on the fly from Wx and dWx
 * (ssqueeze_fast, algos.py:126-150). Sfs (na) non-NULL selects the STFT
 * phase transform |Sfs_i - Im(dS/S)/2pi| (algos.py:956-984). */
SSQB_API int ssqb_ssqueeze_fast(const void* Wx, const void* dWx, const double* Sfs,
                       const double* row_weights, const ssqb_bins* bins, double gamma,
                       int B, int na, int N, int precision, void* Tx, void* stream);

/* Squeeze from a precomputed phase transform w (inf = skip)
 * (indexed_sum_onfly, algos.py:153-250). */
SSQB_API int ssqb_indexed_sum(const void* Wx, const void* w, const double* row_weights,
                     const ssqb_bins* bins, int B, int na, int N, int precision,
                     void* Tx, void* stream);

/* Fused STFT (replaces _stft.py:127-181 with derivative=True and the
 * phase transform of algos.py:784-816): x (B, N); window and diff_window
 * (n_fft) double, diff_window already scaled as the reference does (times
 * fs when modulated); Sfs (n_fft/2+1) double. Outputs (B, n_fft/2+1,
 * n_frames), n_frames = (N-1)/hop + 1; dSx, w, idx optional. n_fft is a
 * power of two <= 4096, or any length in [4, 1024] (Bluestein's chirp-z
 * transform through a power-of-two length >= 2 n_fft - 1, float64
 * arithmetic); n1 is the left pad of the N + n_fft - 1 padding. */
SSQB_API int ssqb_stft(const void* x, int B, int N, int n_fft, int hop, int n1, int padtype,
              int modulated, const double* window, const double* diff_window,
              const double* Sfs, const ssqb_bins* bins, double gamma, int precision,
              void* Sx, void* dSx, void* w, uint16_t* idx, int idx_pitch, void* stream);

/* ssqb_cwt without a caller workspace, for callers that cannot allocate
 * device memory on their call path: for example a plugin inside a host
 * application that reserves all device memory for its own allocator, or a
 * streaming loop that cannot afford the implicit device synchronization of
 * cudaMalloc. No counterpart in ssqueezepy (the reference always allocates
 * through torch / CuPy).
 *
 * Arguments and outputs are those of ssqb_cwt (the caller still provides x,
 * scales, Wx, idx, ...); the padded-signal spectrum and the two-pass
 * intermediate live in one fixed scratch array of ssqb_cwt_noalloc_max_bytes()
 * (16 MiB) of module memory that every device loading the library holds
 * until the process exits. A call needs B * Npad * 16 bytes for Npad <= 2048;
 * above that B * Npad * 48 bytes with float64 arithmetic (SSQB_F64,
 * SSQB_F32X) and B * Npad * 32 bytes with SSQB_F32. A call needing more
 * fails with SSQB_EINVAL and a message naming the size; the exact figure is
 * the minimum ssqb_cwt would accept, and ssqb_cwt_noalloc_max_bytes() gives
 * the limit. The first call on a device
 * looks up the array's device address (and builds the twiddle tables); make
 * that first call before any stream capture. Nothing is allocated or freed.
 * All calls share the one array: calls that overlap on the GPU (other
 * streams, other host threads) race and corrupt each other's results; issue
 * them on one stream or otherwise order them. Nothing in the array needs to
 * start at zero: each call writes every element it later reads. */
SSQB_API int ssqb_cwt_noalloc(const void* x, int B, int N, int Npad, int n1, int padtype,
                              int rpadded, const double* scales, int na,
                              const ssqb_wavelet* wavelet, double dt, const ssqb_bins* bins,
                              double gamma, int precision, void* Wx, void* dWx, void* w,
                              uint16_t* idx, int idx_pitch, void* stream);

/* Size of the fixed scratch array of ssqb_cwt_noalloc, in bytes. */
SSQB_API size_t ssqb_cwt_noalloc_max_bytes(void);

/* One-integral inverse CWT as a weighted row sum (_cwt.py:479-482 with the
 * scaling of :441-452): x[b, j] = sum_i Re(Wx[b, i, j]) * row_weights[i]
 * + x_mean[b] * mean_weight. x (B, N) real of the given precision; x_mean
 * (B) double, may be NULL. */
SSQB_API int ssqb_icwt(const void* Wx, const double* row_weights, const double* x_mean,
                       double mean_weight, int B, int na, int N, int precision,
                       void* x, void* stream);

/* Inverse synchrosqueeze (issq_cwt, _ssq_cwt.py:313-400; issq_stft,
 * _ssq_stft.py:139-198): Tx (nrows, N) complex; with K = 0, x (N) =
 * scale * sum_k Re Tx[k, :]; with K components (K <= 16), cc and cw (N, K)
 * int32 (device) give per column the row range [clip(cc - cw), clip(cc + cw)]
 * (clipped to [0, nrows], empty where cc = -1) and x (K + 1, N) float64
 * holds each component's range sum and, last, the sum of the rows outside
 * every range, all times scale. With K = 0, x has the real type of the
 * precision. scale = 2 / Css for the CWT, 2 / window[n_fft / 2] for
 * the STFT. Float64 accumulation. */
SSQB_API int ssqb_issq(const void* Tx, int nrows, int N, const int32_t* cc, const int32_t* cw,
                       int K, double scale, int precision, void* x, void* stream);

/* Time-frequency ridge extraction (ridge_extraction.py:11-232, its serial
 * code path): Tf (nf, N) complex; s (nf) the frequency axis the jump
 * penalty uses (log scales for the CWT, frequencies for the STFT) and
 * scales (nf) the values reported per ridge, both of the precision's real
 * type (device); penalty, eps and the arithmetic in that type (float32 for
 * SSQB_F32 / SSQB_F32X). For each of n_ridges ridges: E = -log(|Tf|^2 /
 * column max + eps), forward accumulation of min(E + penalty * ds^2) over
 * time, backward re-tracking within eps, then rows [r - bw, r + bw) of
 * the energy (Python slice rules) are cleared. Outputs (N, n_ridges):
 * ridge_idx int32, ridge_f and ridge_e (real, optional). */
SSQB_API size_t ssqb_ridges_workspace_bytes(int nf, int N, int precision);
SSQB_API int ssqb_extract_ridges(const void* Tf, int nf, int N, const void* s,
                                 const void* scales, double penalty, int n_ridges, int bw,
                                 double eps, int precision, int32_t* ridge_idx, void* ridge_f,
                                 void* ridge_e, void* workspace, size_t workspace_bytes,
                                 void* stream);

/* ---- batches of signals of uneven length ---------------------------------
 * ssqueezepy transforms a 2D input of equal-length rows (_cwt.py:270-271) and
 * squeezes it one signal at a time (ssqueezing.py:210-214); signals of
 * different lengths need one call each. These entry points take many
 * signals at once, packed end to end, each described by an ssqb_sig.
 * Offsets count elements of the packed arrays. All signals of one
 * ssqb_cwt_batch call share the padded length Npad (group them by
 * p2up(N), utils/common.py:32-51); ssqb_squeeze_batch takes any mix. */
typedef struct ssqb_sig {
  int64_t x_off;          /* first sample of the signal in x */
  int64_t out_off;        /* first element of its (na, N) block in Wx and Tx */
  int64_t idx_off;        /* first element of its (na, idx_pitch) block in idx */
  const double* scales;   /* device, (na) float64 */
  const double* weights;  /* device, (na) float64 squeeze row weights */
  int32_t N, n1, na, idx_pitch;
  int32_t mode, idx1, flipud, nbins;  /* bin mapping as in ssqb_bins; nbins = na */
  double p[4];
} ssqb_sig;

/* Workspace bytes of ssqb_cwt_batch: the float64 spectra of all nsig
 * signals plus a bounded intermediate (signals are processed in chunks that
 * fit it). */
SSQB_API size_t ssqb_cwt_batch_workspace_bytes(int nsig, int Npad, int precision);

/* ssqb_cwt with bin index for nsig float32 signals of one padded length:
 * x packed float32; Wx complex64 and idx uint16 written at each signal's
 * offsets. `sigs` is a host array of the descriptors, used to check the
 * arguments and size the launches; `sigs_dev` holds the same descriptors in
 * device memory and is what the kernels read. precision SSQB_F32 or
 * SSQB_F32X. A CUDA graph may capture the call once one call has run on the
 * device. */
SSQB_API int ssqb_cwt_batch(const float* x, const ssqb_sig* sigs, const ssqb_sig* sigs_dev,
                            int nsig, int Npad, int padtype, const ssqb_wavelet* wavelet,
                            double dt, double gamma, int precision, void* Wx, uint16_t* idx,
                            void* workspace, size_t workspace_bytes, void* stream);

/* Number of kernel launches of one ssqb_cwt_batch call with these
 * descriptors (host array) and workspace size; -1 on bad arguments. Queries
 * the current device's SM count; no reference counterpart. */
SSQB_API int ssqb_cwt_batch_launches(const ssqb_sig* sigs, int nsig, int Npad, int precision,
                                     size_t workspace_bytes);

/* ssqb_cwt_batch with rows band_from and on (of every signal that has them)
 * through the band-limited single pass at 2^band_log bins (see ssqb_cwt_ex);
 * every signal's rows from band_from must have wavelet bands of at most that
 * many bins (ssqb_cwt_band_rows gives both figures for one signal's scales;
 * a batch takes the largest band_from and band_log of its signals; a row
 * found wider on the device sets the status word). band_from >= the largest
 * na: ssqb_cwt_batch. No reference counterpart. */
SSQB_API int ssqb_cwt_batch_ex(const float* x, const ssqb_sig* sigs, const ssqb_sig* sigs_dev,
                               int nsig, int Npad, int padtype, const ssqb_wavelet* wavelet,
                               double dt, double gamma, int precision, void* Wx,
                               uint16_t* idx, void* workspace, size_t workspace_bytes,
                               int band_from, int band_log, void* stream);

/* Launches of one ssqb_cwt_batch_ex call. */
SSQB_API int ssqb_cwt_batch_ex_launches(const ssqb_sig* sigs, int nsig, int Npad,
                                        int precision, size_t workspace_bytes, int band_from,
                                        int band_log);

/* The rows of a CWT with these host scales that ssqb_cwt_ex sends through the
 * band-limited single pass: the first such row (`band_from`, na if none; the
 * rest of the rows are such too) and the power of two of their largest band
 * (`band_log`, 0 if none). max_bins: the largest band length allowed (a power
 * of two of at most half a tile; 0 = the ssqb_cwt_ex default for this
 * Npad). No reference counterpart. */
SSQB_API int ssqb_cwt_band_rows(const double* scales_host, int na, int Npad,
                                const ssqb_wavelet* wavelet, int precision, int max_bins,
                                int* band_from, int* band_log);

/* ssqb_squeeze over nsig signals of any lengths, one launch: Tx (complex64)
 * at each signal's out_offset, from its Wx block, idx block and weights. */
SSQB_API int ssqb_squeeze_batch(const void* Wx, const uint16_t* idx, const ssqb_sig* sigs,
                                const ssqb_sig* sigs_dev, int nsig, int precision, void* Tx,
                                void* stream);

/* ---- adjoints, for reverse-mode differentiation ----------------------------
 * ssqueezepy has no backward pass; its only differentiable piece is torch
 * autograd through its torch-based GPU `cwt` (_cwt.py:250-311 on torch
 * tensors). These entry points are the transposes of the forward maps, with
 * bins held fixed (piecewise constant). Gradients follow torch's complex
 * convention, g = dL/dRe + i dL/dIm. precision: SSQB_F32 / SSQB_F32X (float32
 * data and arithmetic) or SSQB_F64. accumulate != 0 adds to the output
 * instead of overwriting it. */

/* Workspace bytes of ssqb_cwt_adjoint (spectrum accumulator, real inverse
 * and a bounded chunk of rows). */
SSQB_API size_t ssqb_cwt_adjoint_workspace_bytes(int B, int Npad, int na, int precision);

/* Gradient of x through Wx = cwt(x) (the transposed CWT: per row a forward
 * FFT of the gradient placed at the signal's padded columns, times psih,
 * summed over rows, one inverse FFT, then the transpose of the padding). The
 * gradient of Wx is the sum of up to three sources, each optional:
 *   gWx (B, na, N) complex                          direct
 *   gTx (B, nbins, N) complex through idx           c_i gTx[idx[i, j], j]
 *     (idx (B, na, idx_pitch) from the forward, sq_weights c (na))
 *   gxr (B, N) real through the icwt row weights    w_i gxr[j]
 * so a whole ssq_cwt + icwt backward needs no (na, N) buffer. Output gx
 * (B, N) real. Geometry and wavelet as in ssqb_cwt; padtype 3 (replicate) is
 * SSQB_EUNSUPPORTED. */
SSQB_API int ssqb_cwt_adjoint(const void* gWx, const void* gTx, const uint16_t* idx,
                              int idx_pitch, const double* sq_weights, int nbins,
                              const void* gxr, const double* icwt_weights, int B, int N,
                              int Npad, int n1, int padtype, const double* scales, int na,
                              const ssqb_wavelet* wavelet, int precision, void* gx,
                              int accumulate, void* workspace, size_t workspace_bytes,
                              void* stream);

/* Workspace bytes of ssqb_stft_adjoint: the real per-frame inverse
 * transforms, B * n_fft * n_frames elements of the data precision. */
SSQB_API size_t ssqb_stft_adjoint_workspace_bytes(int B, int N, int n_fft, int hop,
                                                  int precision);

/* Gradient of x through Sx = stft(x) (the transposed STFT of ssqb_stft's
 * framing, window and one-sided FFT): per frame the real part of the
 * inverse transform of the one-sided gradient, times the window, added back
 * at the frame's samples, then the transpose of the padding. The gradient of
 * Sx is gSx (B, n_fft/2+1, n_frames) and / or, through the squeeze, gTx with
 * the forward's idx and sq_weights (as in ssqb_cwt_adjoint). window is the
 * forward's (n_fft) window (double, device); geometry as in ssqb_stft. */
SSQB_API int ssqb_stft_adjoint(const void* gSx, const void* gTx, const uint16_t* idx,
                               int idx_pitch, const double* sq_weights, int B, int N,
                               int n_fft, int hop, int n1, int padtype, int modulated,
                               const double* window, int precision, void* gx, int accumulate,
                               void* workspace, size_t workspace_bytes, void* stream);

/* Phase transform by differences along time (difftype 'phase' and
 * 'numeric' of ssq_cwt / phase_cwt). Each of the B*na rows of Wx is ncol
 * wide; the transform reads columns col0 .. col0+M-1 and writes w (B, na, M).
 *   mode 1, 'phase' (_ssq_cwt.py:490-496): w[j] = |u[j+1] - u[j]| / 2pi for
 *     j < M-1 and |u[M-1] - u[0]| / 2pi, u the angle of Wx unwrapped along
 *     time (numpy unwrap: steps of size pi or more moved into [-pi, pi]);
 *   mode 2, 'numeric' (phase_cwt_num, _ssq_cwt.py:512-586): w = |Im(D/Wx)| /
 *     2pi, D the difference of order `difforder` (1 forward, 2 second-order
 *     forward, 4 central) over dt, periodic within the M columns;
 * w = inf where |Wx| < gamma. Arithmetic in float64 for either precision. */
SSQB_API int ssqb_phase_diff(const void* Wx, int B, int na, int ncol, int col0, int M,
                             int mode, int difforder, double dt, double gamma,
                             int precision, void* w, void* stream);

/* Workspace bytes of ssqb_trigdiff: the spectra of a chunk of rows (up to
 * 256 MB of them, at least one row) and the two-pass intermediate. */
SSQB_API size_t ssqb_trigdiff_workspace_bytes(int rows, int Npad);

/* Frequency-domain derivative of rows (trigdiff, utils/common.py:161-245):
 * D = ifft(fft(Ap) * i xi fs), xi_k = 2 pi kk / Npad with kk = k for
 * k <= Npad/2 and k - Npad above (no Nyquist halving), Ap = A padded to Npad
 * with n1 samples on the left by padtype (5 = none: A is already Npad long,
 * n1 = 0). out (rows, N_out) = D[:, out_off : out_off + N_out]. A and out
 * complex of the data precision; float64 arithmetic. Npad a power of two in
 * [8, 2^22]. */
SSQB_API int ssqb_trigdiff(const void* A, int rows, int M, int Npad, int n1, int padtype,
                           double fs, int out_off, int N_out, int precision, void* out,
                           void* workspace, size_t workspace_bytes, void* stream);

/* Workspace bytes of ssqb_istft: the real frames, B * n_fft * n_frames
 * elements of the data precision. */
SSQB_API size_t ssqb_istft_workspace_bytes(int B, int n_fft, int n_frames, int precision);

/* Inverse STFT (istft, _stft.py:184-256): per frame the inverse real FFT of
 * Sx's column (n_fft/2+1 bins; the imaginary parts of the DC and Nyquist bins
 * are ignored), fftshifted when modulated, overlap-added at hop with
 * wa = window^win_exp (utils/stft_utils.py:141-182), divided by the window
 * norm sum_{t < (N-1)/hop+1} w1[p - t hop], w1 = window^(win_exp+1)
 * (utils/stft_utils.py:169-191), where the norm exceeds `tiny` (the smallest
 * normal number of the data type, _stft.py:245-250), and unpadded by
 * n_fft/2 samples on the left. Sx (B, n_fft/2+1, n_frames); wa, w1 (n_fft)
 * double; x (B, N) real. The frames must end inside the padded signal:
 * (n_frames - 1) * hop <= N - 1. n_fft a power of two <= 4096, or any length
 * in [4, 1024] (the frames by Bluestein's chirp-z transform, float64). */
SSQB_API int ssqb_istft(const void* Sx, int B, int n_fft, int n_frames, int hop, int N,
                        int modulated, const double* wa, const double* w1, double tiny,
                        int precision, void* x, void* workspace, size_t workspace_bytes,
                        void* stream);

/* Gradient of Wx through the squeeze, a gather through the bin index:
 * gWx[b, i, j] = row_weights[i] * gTx[b, idx[b, i, j], j] (0 where idx is
 * 0xFFFF). Transpose of ssqb_squeeze. */
SSQB_API int ssqb_squeeze_adjoint(const void* gTx, const uint16_t* idx, int idx_pitch,
                                  const double* row_weights, int B, int na, int N, int nbins,
                                  int precision, void* gWx, int accumulate, void* stream);

/* Gradient of Wx through the one-integral icwt: gWx[b, i, j] =
 * row_weights[i] * gx[b, j] (real). Transpose of ssqb_icwt. */
SSQB_API int ssqb_icwt_adjoint(const void* gx, const double* row_weights, int B, int na,
                               int N, int precision, void* gWx, int accumulate, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SSQB_H_ */
