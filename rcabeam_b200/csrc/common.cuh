// Shared device helpers for the rcabeam B200 kernels: complex arithmetic,
// float64 RCA geometry, and the mbarrier / TMA primitives of the staged
// pipelines.  Every spin-wait here is bounded: after kWaitLimitNs of global
// time it records an error code in a device word and reports failure, so a
// kernel never hangs the GPU.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "rcabeam.h"

namespace rcb {

// ---------------------------------------------------------------- complex --
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
// x / sqrt(|x|), zero at zero: the signed square root of the FMAS / DMAS beamformers.
__device__ __forceinline__ float2 csroot(float2 a) {
  float m = hypotf(a.x, a.y);
  float s = m > 0.f ? rsqrtf(m) : 0.f;
  return make_float2(a.x * s, a.y * s);
}
// acc += p * v with the rotation and accumulation fused.
__device__ __forceinline__ float2 cmac(float2 p, float2 v, float2 acc) {
  return make_float2(fmaf(-p.y, v.y, fmaf(p.x, v.x, acc.x)), fmaf(p.y, v.x, fmaf(p.x, v.y, acc.y)));
}

// ---------------------------------------------------------------- geometry --
// One interpolation tap of the RCA delay-and-sum: sample row i0 (negative when
// the voxel/element pair contributes nothing), fractional weight w toward row
// i0 + 1, and the demodulation rotation exp(+j 2 pi fd tau).
struct Tap {
  int i0;
  float w;
  float2 phase;
};

// Receive delay sqrt(z^2 + (v - e)^2) / c with v = x (RC) or y (CR) and the
// f-number aperture |v - e| <= z / (2 fn).  The float64 operation order (two
// rounded products, a rounded sum, a correctly rounded sqrt and quotient)
// matches the float64 oracle so that taps on exact sample boundaries agree.
__device__ __forceinline__ double receive_delay(double v, double z, double e, double c, double fn, bool* active) {
  double d = __dadd_rn(v, -e);
  double r = __dsqrt_rn(__dadd_rn(__dmul_rn(z, z), __dmul_rn(d, d)));
  *active = fn <= 0.0 || fabs(d) <= __ddiv_rn(z, __dmul_rn(2.0, fn));
  return __ddiv_rn(r, c);
}

// Transmit delay (z cos(theta) + u sin(theta)) / c with u = y (RC) or x (CR).
__device__ __forceinline__ double transmit_delay(double u, double z, double cs, double sn, double c) {
  return __ddiv_rn(__dadd_rn(__dmul_rn(z, cs), __dmul_rn(u, sn)), c);
}

// sample = (tau - start) fs; valid iff 0 <= sample <= ns - 1 (reference sim.py:379-380).
// The phase is reduced in float64 (fd tau minus its nearest integer) before the
// float32 sincospi, so its error stays near 1e-7 rad at any depth.
__device__ __forceinline__ Tap make_tap(double tau, double start, double fs, double fd, int ns, bool active) {
  Tap t;
  double sample = __dmul_rn(__dadd_rn(tau, -start), fs);
  if (!active || !(sample >= 0.0) || !(sample <= double(ns - 1))) {
    t.i0 = -1;
    t.w = 0.f;
    t.phase = make_float2(0.f, 0.f);
    return t;
  }
  double fl = floor(sample);
  t.i0 = int(fl);
  t.w = float(sample - fl);
  double cyc = fd * tau;
  cyc -= rint(cyc);
  float s, co;
  sincospif(2.0f * float(cyc), &s, &co);
  t.phase = make_float2(co, s);
  return t;
}

// ---------------------------------------------------------- bounded waits --
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s
enum DeviceError : int { kErrNone = 0, kErrWaitFull = 1, kErrWaitEmpty = 2, kErrWaitDrain = 3 };

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity; false (and *err set) after `limit_ns`.
__device__ __noinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code,
                                       unsigned long long limit_ns = kWaitLimitNs) {
  if (mbar_test(bar, parity)) return true;
  unsigned long long start = global_ns();
  for (uint32_t i = 0;; ++i) {
    if (mbar_test(bar, parity)) return true;
    if ((i & 255u) == 255u && global_ns() - start > limit_ns) {
      if (err) atomicCAS(err, 0, code);
      return false;
    }
  }
}

// Failure-path check of the bounded waits: every warp of one CTA waits, with
// `limit_ns`, on an mbarrier that nothing arrives on, exactly as a pipeline
// stage whose producer never delivers.  Each wait gives up, records `code` in
// the device error word and the kernel returns; *gave_up counts the waits that
// returned false.
__global__ void wait_selftest(int* err, int code, unsigned long long limit_ns, int* gave_up) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0 && !mbar_wait(&bar, 0, err, code, limit_ns)) atomicAdd(gave_up, 1);
}

// mbar_wait with the already-complete case inline (no call on the fast path).
__device__ __forceinline__ bool mbar_wait_fast(uint64_t* bar, uint32_t parity, int* err, int code) {
  return mbar_test(bar, parity) || mbar_wait(bar, parity, err, code);
}

// 2-D tiled TMA load into this CTA's shared memory, completing on an mbarrier.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

// 3-D tiled TMA load into this CTA's shared memory, completing on an mbarrier.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// 4-D tiled TMA load into this CTA's shared memory, completing on an mbarrier.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ------------------------------------------------------------------ host --
inline rcabeam_status launch_status() {
  return cudaGetLastError() == cudaSuccess ? RCABEAM_SUCCESS : RCABEAM_ERROR_CUDA;
}

}  // namespace rcb
