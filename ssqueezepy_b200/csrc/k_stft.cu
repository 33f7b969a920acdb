// Fused STFT tile kernels (one pass; power-of-two n_fft up to one tile).
#include "tile_launch.cuh"

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
  return dispatch_log<3, tile_log<C>()>(log2L, [&](auto k) {
    return launch_stft<Op, C, decltype(k)::value>(op, B, tb, st);
  });
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
