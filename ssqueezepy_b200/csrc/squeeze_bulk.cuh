// Synchrosqueeze with rows streamed through a shared-memory ring by 1-D bulk
// async copies (cp.async.bulk + mbarrier).
//
// One warp owns 32 consecutive columns of one signal and the whole Tx
// column block, nbins x 32 float2, in shared memory. Lane 0 keeps D stages of
// RPS rows (Wx: 32 complex64, idx: 32 uint16 per row) in flight; every lane
// walks the rows of its column in ascending order and adds runs of entries
// that fall in the same bin in a register before one read-modify-write of
// the accumulator, so the fixed row order of the reference's per-column loop
// (algos.py:879-895) is kept up to the grouping of each run's additions:
// deterministic, no atomics.
//
// Requirements (checked by the launcher): float32 data, N even (Wx rows then
// start on 16-byte boundaries), idx row pitch a multiple of 32 columns.
// Every mbarrier wait is bounded; on expiry the kernel records
// DEV_TIMEOUT, drains its copies in flight (bounded) and returns.
#pragma once
#include "ssqb_ops.cuh"

namespace ssqb {

constexpr int kSqRPS = 8;   // rows per stage
constexpr int kSqD = 6;     // stages in flight
constexpr uint32_t kSqSpin = 1u << 22;  // try_wait attempts before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; false when the attempts ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kSqSpin; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

struct SqRing {
  float2 wx[kSqD][kSqRPS][32];
  uint16_t ix[kSqD][kSqRPS][32];
  uint64_t bar[kSqD];
};

__global__ void __launch_bounds__(32)
squeeze_bulk_kernel(const float2* __restrict__ Wx, const uint16_t* __restrict__ idx,
                    int idx_pitch, const double* __restrict__ cst, int na, int N, int nbins,
                    float2* __restrict__ Tx, int* status) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SqRing& ring = *reinterpret_cast<SqRing*>(smem_raw);
  float2* acc = reinterpret_cast<float2*>(smem_raw + sizeof(SqRing));  // [nbins][32]
  float* cs = reinterpret_cast<float*>(acc + (size_t)nbins * 32);       // [na]
  const int lane = threadIdx.x;
  const int b = blockIdx.y;
  const int j0 = blockIdx.x * 32;
  const int ncol = min(32, N - j0);
  const bool live = lane < ncol;
  const int nstages = (na + kSqRPS - 1) / kSqRPS;
  const float2* wbase = Wx + (size_t)b * na * N + j0;
  const uint16_t* ibase = idx + (size_t)b * na * idx_pitch + j0;
  const uint32_t wbytes = (uint32_t)ncol * 8u;  // multiple of 16 (N even)

  auto issue = [&](int s) {  // lane 0 only
    const int slot = s % kSqD;
    const int r0 = s * kSqRPS;
    const int nr = min(kSqRPS, na - r0);
    mbar_expect_tx(&ring.bar[slot], (uint32_t)nr * (wbytes + 64u));
    for (int r = 0; r < nr; ++r) {
      bulk_g2s(&ring.wx[slot][r][0], wbase + (size_t)(r0 + r) * N, wbytes, &ring.bar[slot]);
      bulk_g2s(&ring.ix[slot][r][0], ibase + (size_t)(r0 + r) * idx_pitch, 64u,
               &ring.bar[slot]);
    }
  };

  if (lane == 0) {
    for (int s = 0; s < kSqD; ++s) mbar_init(&ring.bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (lane == 0)
    for (int s = 0; s < min(kSqD, nstages); ++s) issue(s);
  for (int k = lane; k < nbins * 32; k += 32) acc[k] = make_float2(0.f, 0.f);
  for (int i = lane; i < na; i += 32) cs[i] = (float)cst[i];
  __syncwarp();

  int kcur = -1;
  float2 run = make_float2(0.f, 0.f);
  int sfail = -1;
  int issued = min(kSqD, nstages);
  for (int s = 0; s < nstages; ++s) {
    const int slot = s % kSqD;
    if (!mbar_wait(&ring.bar[slot], (uint32_t)((s / kSqD) & 1))) {
      sfail = s;
      break;
    }
    const int r0 = s * kSqRPS;
    const int nr = min(kSqRPS, na - r0);
#pragma unroll
    for (int r = 0; r < kSqRPS; ++r) {
      if (r < nr && live) {
        const uint16_t k16 = ring.ix[slot][r][lane];
        if (k16 != kNoBin) {
          const int k = (int)k16;
          if (k >= nbins) {
            set_status(status, DEV_BAD_BIN);
          } else {
            const float2 v = ring.wx[slot][r][lane];
            const float c = cs[r0 + r];
            if (k != kcur) {
              if (kcur >= 0) {
                float2& a = acc[kcur * 32 + lane];
                a.x += run.x;
                a.y += run.y;
              }
              kcur = k;
              run = make_float2(v.x * c, v.y * c);
            } else {
              run.x = fmaf(v.x, c, run.x);
              run.y = fmaf(v.y, c, run.y);
            }
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0 && issued < nstages) {
      // the slot's rows are in registers / consumed: order those generic-proxy
      // reads before the async-proxy writes of the next copy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(issued);
    }
    issued = __shfl_sync(0xffffffffu, issued + (issued < nstages ? 1 : 0), 0);
  }
  if (sfail >= 0) {
    // drain the copies still in flight before the CTA's shared memory goes away
    set_status(status, DEV_TIMEOUT);
    if (lane == 0)
      for (int s = sfail; s < issued; ++s)
        mbar_wait(&ring.bar[s % kSqD], (uint32_t)((s / kSqD) & 1));
    __syncwarp();
    return;
  }
  if (kcur >= 0) {
    float2& a = acc[kcur * 32 + lane];
    a.x += run.x;
    a.y += run.y;
  }
  __syncwarp();
  if (live) {
    float2* out = Tx + (size_t)b * nbins * N + j0 + lane;
    for (int k = 0; k < nbins; ++k) out[(size_t)k * N] = acc[k * 32 + lane];
  }
}

}  // namespace ssqb
