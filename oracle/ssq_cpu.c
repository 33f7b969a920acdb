/* CPU restatement of the reference's column-parallel squeeze kernels, for
 * the timed CPU arm. TEST INFRASTRUCTURE ONLY: loaded by oracle/ssq_cpu_path.py
 * (bench.py's reference arm and CPU baseline); the product never uses it.
 *
 * It follows ssqueezepy's numba kernels _ssq_cwt_log_piecewise_par
 * (algos.py:879-895) and _ssq_cwt_log_par (algos.py:913-924): columns in
 * parallel (numba prange -> OpenMP), rows in ascending order within a
 * column; complex64 data; the phase transform's numerator in float32 and its
 * denominator promoted to float64 by the literal 6.283185307179586, as numba
 * evaluates it; bins by round-half-to-even (numba's round); Tx[k, j] +=
 * Wx[i, j] * const[i] in complex64.
 *
 * Build: gcc -O3 -fopenmp -shared -fPIC oracle/ssq_cpu.c -o oracle/_lib/libssqcpu.so
 */
#include <math.h>

/* mode 0: log bins (vlmin0, dvl0); mode 1: log-piecewise (vlmin0, vlmin1,
 * dvl0, dvl1, idx1). Wx, dWx: (na, ld) interleaved complex64, columns
 * [0, N) used (the unpadded view of the padded transform); Tx: (na, N),
 * must start at zero. */
void ssq_cpu_squeeze(const float* Wx, const float* dWx, float* Tx, const float* cst,
                     int na, int N, long long ld, double gamma, int mode, double vlmin0,
                     double vlmin1, double dvl0, double dvl1, int idx1, int omax,
                     int flipud) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < N; ++j) {
    for (int i = 0; i < na; ++i) {
      const long long o = 2LL * ((long long)i * ld + j);
      const float C = Wx[o], D = Wx[o + 1];
      if (hypotf(C, D) > gamma) {
        const float A = dWx[o], B = dWx[o + 1];
        const float num = B * C - A * D;
        const double w = fabs((double)num / ((double)(C * C + D * D) * 6.283185307179586));
        const double wl = log2(w);
        int k;
        if (mode == 1 && wl > vlmin1) {
          const double r = nearbyint((wl - vlmin1) / dvl1) + idx1;
          k = (int)(r < omax ? r : omax);
        } else if (mode == 1) {
          const double r = nearbyint((wl - vlmin0) / dvl0);
          k = (int)(r > 0 ? r : 0);
        } else {
          double r = nearbyint((wl - vlmin0) / dvl0);
          r = r > 0 ? r : 0;
          k = (int)(r < omax ? r : omax);
        }
        if (flipud) k = omax - k;
        const long long t = 2LL * ((long long)k * N + j);
        Tx[t] += C * cst[i];
        Tx[t + 1] += D * cst[i];
      }
    }
  }
}
