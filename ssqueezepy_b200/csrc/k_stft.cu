// Fused STFT tile kernels (one pass; power-of-two n_fft up to one tile).
#include "launch.h"

namespace ssqb {

template <class Op, typename C, int LOGL>
static int launch_stft(const Op& op, int B, const Tables& tb, cudaStream_t st) {
  constexpr int NF = tile_of<C>() / (1 << LOGL);
  const size_t smem = tile_smem<C>(Op::NARR, LOGL);
  auto k = tile_single<Op, C, LOGL, -1>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  dim3 grid((op.nframes + NF - 1) / NF, 1, B);
  k<<<grid, kNT, smem, st>>>(op, tb);
  return cudaGetLastError();
}

template <class Op, typename C>
static int run_stft(const Op& op, int B, int log2L, const Tables& tb, cudaStream_t st) {
  switch (log2L) {
    case 3: return launch_stft<Op, C, 3>(op, B, tb, st);
    case 4: return launch_stft<Op, C, 4>(op, B, tb, st);
    case 5: return launch_stft<Op, C, 5>(op, B, tb, st);
    case 6: return launch_stft<Op, C, 6>(op, B, tb, st);
    case 7: return launch_stft<Op, C, 7>(op, B, tb, st);
    case 8: return launch_stft<Op, C, 8>(op, B, tb, st);
    case 9: return launch_stft<Op, C, 9>(op, B, tb, st);
    case 10: return launch_stft<Op, C, 10>(op, B, tb, st);
    case 11: return launch_stft<Op, C, 11>(op, B, tb, st);
    case 12:
      if constexpr (tile_of<C>() >= 4096) return launch_stft<Op, C, 12>(op, B, tb, st);
      else return (int)cudaErrorInvalidValue;
    default: return (int)cudaErrorInvalidValue;
  }
}

int run_stft_f32(const StftOp<float, float2>& op, int B, int log2L, const Tables& tb,
                 cudaStream_t st) {
  return run_stft<StftOp<float, float2>, float2>(op, B, log2L, tb, st);
}

int run_stft_f64(const StftOp<double, double2>& op, int B, int log2L, const Tables& tb,
                 cudaStream_t st) {
  return run_stft<StftOp<double, double2>, double2>(op, B, log2L, tb, st);
}

int run_stft_f32x(const StftOp<float, double2, float2>& op, int B, int log2L,
                  const Tables& tb, cudaStream_t st) {
  return run_stft<StftOp<float, double2, float2>, double2>(op, B, log2L, tb, st);
}

}  // namespace ssqb
