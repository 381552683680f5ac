// Channel packing: (samples, channels, angles, frames) -> (channels, angles,
// samples, frames), frames innermost on both sides (reference ensemble.cu:119-141).
// The transpose permutes whole frame rows, so each warp copies one row with
// coalesced loads and stores; it is HBM-bound (2 x input bytes).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace rcb {

constexpr int kPackThreads = 256;

// One warp per (channel, angle, sample) row of nt frames.
template <bool HALF>
__global__ void __launch_bounds__(kPackThreads)
    pack_rows(const float2* __restrict__ src, void* __restrict__ dst, int* __restrict__ range_error, size_t ns,
              size_t nc, size_t na, size_t nt) {
  const size_t rows = ns * nc * na;
  const size_t warps = size_t(gridDim.x) * (kPackThreads / 32);
  const int lane = threadIdx.x & 31;
  bool bad = false;
  for (size_t row = size_t(blockIdx.x) * (kPackThreads / 32) + threadIdx.x / 32; row < rows; row += warps) {
    // Target row index is (c * na + a) * ns + s.
    size_t s = row % ns;
    size_t ca = row / ns;
    size_t a = ca % na;
    size_t c = ca / na;
    const float2* in = src + ((s * nc + c) * na + a) * nt;
    if constexpr (HALF) {
      __half2* out = static_cast<__half2*>(dst) + row * nt;
      for (size_t t = lane; t < nt; t += 32) {
        float2 v = __ldg(in + t);
        bad |= !isfinite(v.x) || !isfinite(v.y) || fabsf(v.x) > 65504.f || fabsf(v.y) > 65504.f;
        out[t] = __floats2half2_rn(v.x, v.y);
      }
    } else {
      float2* out = static_cast<float2*>(dst) + row * nt;
      for (size_t t = lane; t < nt; t += 32) out[t] = __ldg(in + t);
    }
  }
  if constexpr (HALF) {
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(range_error, 1);
  }
}

// (s, c, a, t) complex64 -> two (c, a, s, t) planes of BF16 (re, im) pairs:
// hi = bf16(x), lo = bf16(x - hi), so hi + lo keeps ~16 significant bits.
// Non-finite components set *range_error.
__global__ void __launch_bounds__(kPackThreads)
    pack_split_rows(const float2* __restrict__ src, __nv_bfloat162* __restrict__ hi, __nv_bfloat162* __restrict__ lo,
                    int* __restrict__ range_error, size_t ns, size_t nc, size_t na, size_t nt) {
  const size_t rows = ns * nc * na;
  const size_t warps = size_t(gridDim.x) * (kPackThreads / 32);
  const int lane = threadIdx.x & 31;
  bool bad = false;
  for (size_t row = size_t(blockIdx.x) * (kPackThreads / 32) + threadIdx.x / 32; row < rows; row += warps) {
    size_t s = row % ns;
    size_t ca = row / ns;
    size_t a = ca % na;
    size_t c = ca / na;
    const float2* in = src + ((s * nc + c) * na + a) * nt;
    for (size_t t = lane; t < nt; t += 32) {
      float2 v = __ldg(in + t);
      bad |= !isfinite(v.x) || !isfinite(v.y);
      __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
      float2 hf = __bfloat1622float2(h);
      hi[row * nt + t] = h;
      lo[row * nt + t] = __floats2bfloat162_rn(v.x - hf.x, v.y - hf.y);
    }
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(range_error, 1);
}

template <bool HALF>
inline rcabeam_status launch_pack(const void* source, void* target, int* range_error, size_t ns, size_t nc,
                                  size_t na, size_t nt) {
  size_t rows = ns * nc * na;
  size_t blocks = (rows + kPackThreads / 32 - 1) / (kPackThreads / 32);
  if (blocks > 148ull * 64ull) blocks = 148ull * 64ull;
  pack_rows<HALF><<<unsigned(blocks), kPackThreads>>>(static_cast<const float2*>(source), target, range_error, ns,
                                                       nc, na, nt);
  return launch_status();
}

}  // namespace rcb
