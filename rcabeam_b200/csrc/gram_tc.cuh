// Tensor-core (tcgen05) temporal Gram matrix of a complex64 Casorati matrix.
//
// The complex64 rows x T matrix X is read as a real rows x 2T float32 matrix Y
// (real and imaginary parts interleaved, no copy).  D = Y^T Y holds the complex
// Gram G = X^H X as
//     G[m][n] = (D[2m][2n] + D[2m+1][2n+1]) + j (D[2m][2n+1] - D[2m+1][2n]),
// so the whole product is one real symmetric GEMM with K = rows.  Only the
// upper triangle of 128 x 128 blocks of D is formed (block b of D is the
// 64-frame tile b of G, the tiling the float64 Gram and its finish kernel use).
//
// Work: the upper blocks (b <= c) are packed into units of up to four output
// blocks that stage at most three 128-column blocks (plan_units: triangles
// {a, b, c} first); every unit runs on `slices` CTAs, each over
// one contiguous range of rows, so the CTAs of one slice read the same rows at
// the same time (one HBM read, the rest from L2).  TMEM holds the unit's four
// 128 x 128 float32 accumulators (512 columns); every kFlushRows rows (and at
// the end of the slice) the epilogue adds them, in float64, to the upper
// triangle with atomics, which bounds the float32 accumulation length.
//
// Precision (both with float32 accumulation):
//   tf32   : operands rounded to nearest TF32 (cvt.rna) -- one MMA per K=8;
//   bf16x3 : operands split into BF16 hi + lo, three MMAs per K=16
//            (Ahi Bhi + Alo Bhi + Ahi Blo).
// Before rounding or splitting every element is multiplied by 2^-e, where 2^e
// bounds the Casorati scale s (max |component|), which keeps the products in
// range exactly as the scaled float64 Gram does; the epilogue applies (2^e/s)^2.
//
// Roles (256 threads, one CTA per SM):
//   warp 0       TMA producer: raw float32 boxes (32 columns x 16 rows;
//                SWIZZLE_128B_ATOM_32B for TF32, SWIZZLE_128B for 3xBF16) of
//                the unit's staged blocks into the staging ring;
//   warp 1       TMEM allocator; lane 0 issues tcgen05.mma and commits;
//   warps 2-7    converters: TF32 rounds the staged floats in place (the
//                layouts coincide), so the staging ring is the operand ring
//                (2 x ring stages, eight with three staged blocks); 3xBF16
//                writes hi/lo operands in the UMMA MN-major SWIZZLE_128B
//                layout (ring staging stages and ring operand stages in the
//                same shared memory; ring = 4 with three staged blocks);
//   warps 4-7    also the epilogue (TMEM lane quarters 0-3) at every flush.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "das_tc.cuh"

namespace rcb {
namespace gramtc {

constexpr int kBlock = 128;        // real columns per Gram block (64 complex frames)
constexpr int kRows = 16;          // rows per stage
constexpr int kMaxLoads = 6;       // staged column blocks per unit
constexpr int kMaxTasks = 4;       // output blocks per unit (4 x 128 TMEM columns)
constexpr int kMaxUnits = 48;      // nb <= 16 blocks (T <= 1024): 136 upper blocks -> 43 units
constexpr int kMaxBlocks = 16;
constexpr int kMaxRing = 4;        // deepest 3xBF16 staging and operand rings (TF32: one ring of 2 x ring)
constexpr int kThreads = 256;
constexpr int kConverters = 6 * 32;
constexpr int kSlotBytes = kBlock * kRows * 4;  // 8192: one staged block per stage (f32 or bf16 hi+lo)
// The tensor core rounds each float32 accumulation toward zero (a shrink of
// ~1.3e-8 per update); flushing to float64 every 2048 rows (256 TF32 or 384
// BF16 updates) keeps that bias near 3e-6 of a Gram entry.
constexpr int kFlushRows = 2048;
constexpr int kTmemCols = 512;
// MN-major TF32 operands take the 128-byte swizzle with 32-byte granules (the
// TMA's SWIZZLE_128B_ATOM_32B): 4-row K atoms, so SBO = 512 B; BF16 operands
// take the plain 128-byte swizzle (8-row atoms, SBO = 1024 B).
constexpr uint32_t kLayoutSw128Base32 = 1;

struct Unit {
  int nload;
  int load[kMaxLoads];  // staged block per slot
  int ntask;
  int a_slot[kMaxTasks], b_slot[kMaxTasks];
  int a_blk[kMaxTasks], b_blk[kMaxTasks];
};

struct Params {
  int nunits, slices, nload_max, nt;
  int ring;  // 3xBF16 staging and operand ring depth; TF32 converts in place in one ring of 2 x ring
  long long rows, slice_rows;
  const double* scale;
  double* upper;
  int* err;
  Unit units[kMaxUnits];
};

__host__ __device__ inline size_t smem_bytes(int nload_max, int ring) {
  return size_t(2 * ring) * nload_max * kSlotBytes + 1024 + 1024;
}

// kind::tf32 / kind::f16(BF16) instruction descriptor: F32 accumulate, A and B MN-major.
__host__ __device__ constexpr uint32_t idesc_mn(bool tf32, int m, int n) {
  return (1u << 4) | ((tf32 ? 2u : 1u) << 7) | ((tf32 ? 2u : 1u) << 10) | (1u << 15) | (1u << 16) |
         (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ float round_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo_elem, float hi_elem) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo_elem, hi_elem);
  return *reinterpret_cast<uint32_t*>(&v);
}

// Split 8 scaled floats into BF16 hi and lo 16-byte chunks.
__device__ __forceinline__ void split8(const float (&v)[8], uint4& hi, uint4& lo) {
  float h[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    h[i] = __bfloat162float(__float2bfloat16_rn(v[i]));
    l[i] = v[i] - h[i];
  }
  hi = make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]), pack_bf16(h[6], h[7]));
  lo = make_uint4(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]), pack_bf16(l[4], l[5]), pack_bf16(l[6], l[7]));
}

template <bool TF32>
__global__ void __launch_bounds__(kThreads, 1) gram_tc(const __grid_constant__ CUtensorMap map, const Params p) {
  using namespace rcb::tc;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const Unit& u = p.units[blockIdx.x % p.nunits];
  const int slice = blockIdx.x / p.nunits;
  // TF32: one ring of 2 x ring stages converted in place; 3xBF16: ring staging + ring operand stages.
  const int R = TF32 ? 2 * p.ring : p.ring;
  const size_t stage_bytes = size_t(p.nload_max) * kSlotBytes;
  unsigned char* staging = smem;
  unsigned char* operands = TF32 ? smem : smem + p.ring * stage_bytes;
  uint64_t* stg_full = reinterpret_cast<uint64_t*>(smem + 2 * p.ring * stage_bytes);
  uint64_t* stg_empty = stg_full + R;
  uint64_t* op_full = stg_empty + R;
  uint64_t* op_empty = op_full + R;
  uint64_t* acc_full = op_empty + R;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long r0 = (long long)slice * p.slice_rows;
  const long long r1 = r0 + p.slice_rows < p.rows ? r0 + p.slice_rows : p.rows;
  const int nstages = r1 > r0 ? int((r1 - r0 + kRows - 1) / kRows) : 0;
  constexpr int kStagesPerFlush = kFlushRows / kRows;

  if (threadIdx.x == 0) {
    for (int s = 0; s < R; ++s) {
      mbar_init(&stg_full[s], 1);
      mbar_init(&stg_empty[s], TF32 ? 1 : kConverters / 32);  // TF32: freed by the MMA commit
      mbar_init(&op_full[s], kConverters / 32);
      mbar_init(&op_empty[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 4);
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // Exact power-of-two prescale 2^-e with s = f 2^e, f in [0.5, 1).
  const double s = *p.scale;
  int e = 0;
  if (s > 0.0 && s <= 1.79e308) frexp(s, &e);
  const float prescale = s > 0.0 ? float(ldexp(1.0, -e)) : 1.0f;
  const double factor = s > 0.0 ? (ldexp(1.0, e) / s) * (ldexp(1.0, e) / s) : 1.0;

  if (warp == 0) {
    // ------------------------------------------------------------- producer --
    if (lane == 0) prefetch_tensormap(&map);
    int k = 0;
    bool ok = true;
    for (; k < nstages && ok; ++k) {
      const int s_ = k % R;
      if (k >= R) ok = __all_sync(0xffffffffu, mbar_wait(&stg_empty[s_], ((k / R) - 1) & 1, p.err, kErrWaitEmpty));
      if (!ok) break;
      const int row = int(r0 + (long long)k * kRows);
      if (lane == 0) mbar_arrive_expect_tx(&stg_full[s_], uint32_t(u.nload * kSlotBytes));
      __syncwarp();
      unsigned char* dst = staging + s_ * stage_bytes;
      // 4 boxes (32 columns) per staged block, one box per lane.
      if (lane < 4 * u.nload) {
        const int slot = lane >> 2, box = lane & 3;
        tma_load_2d(dst + slot * kSlotBytes + box * 2048, &map, &stg_full[s_], u.load[slot] * kBlock + 32 * box, row);
      }
    }
    // Drain: the last issued stages' copies have landed before the CTA exits.
    if (lane == 0) {
      for (int d = k - R < 0 ? 0 : k - R; d < k; ++d)
        mbar_wait(&stg_full[d % R], (d / R) & 1, p.err, kErrWaitDrain);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------------------ MMA --
    if (lane == 0) {
      const uint32_t idesc = idesc_mn(TF32, 128, 128);
      int flushes = 0;
      for (int k = 0; k < nstages; ++k) {
        const int s_ = k % R;
        const int in_seg = k % kStagesPerFlush;
        if (in_seg == 0 && flushes > 0 && !mbar_wait(acc_empty, (flushes - 1) & 1, p.err, kErrWaitEmpty)) break;
        if (!mbar_wait(&op_full[s_], (k / R) & 1, p.err, kErrWaitFull)) break;
        tc_fence_after();
        const uint32_t op = smem_u32(operands + s_ * stage_bytes);
        for (int t = 0; t < u.ntask; ++t) {
          const uint32_t d = tmem + uint32_t(kBlock * t);
          if constexpr (TF32) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const uint32_t a = op + u.a_slot[t] * kSlotBytes + q * 1024;
              const uint32_t b = op + u.b_slot[t] * kSlotBytes + q * 1024;
              mma_tf32(d, smem_desc(a, 2048, 512, kLayoutSw128Base32), smem_desc(b, 2048, 512, kLayoutSw128Base32),
                       idesc, (in_seg > 0 || q > 0) ? 1u : 0u);
            }
          } else {
            const uint32_t hi = op, lo = op + uint32_t(p.nload_max) * (kSlotBytes / 2);
            const uint32_t ah = hi + u.a_slot[t] * (kSlotBytes / 2), al = lo + u.a_slot[t] * (kSlotBytes / 2);
            const uint32_t bh = hi + u.b_slot[t] * (kSlotBytes / 2), bl = lo + u.b_slot[t] * (kSlotBytes / 2);
            mma_f16(d, smem_desc(ah, 2048, 1024, kLayoutSw128), smem_desc(bh, 2048, 1024, kLayoutSw128), idesc,
                    in_seg > 0 ? 1u : 0u);
            mma_f16(d, smem_desc(al, 2048, 1024, kLayoutSw128), smem_desc(bh, 2048, 1024, kLayoutSw128), idesc, 1u);
            mma_f16(d, smem_desc(ah, 2048, 1024, kLayoutSw128), smem_desc(bl, 2048, 1024, kLayoutSw128), idesc, 1u);
          }
        }
        mma_commit(TF32 ? &stg_empty[s_] : &op_empty[s_]);
        if (in_seg == kStagesPerFlush - 1 || k == nstages - 1) {
          mma_commit(acc_full);
          ++flushes;
        }
      }
      mma_commit(drain);
      mbar_wait(drain, 0, p.err, kErrWaitDrain);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------ converters / epilogue --
    const int ct = threadIdx.x - 64;  // 0 .. 191
    const bool epilogue = warp >= 4;
    const int quarter = warp & 3;
    int flushes = 0;
    for (int k = 0; k < nstages; ++k) {
      const int s_ = k % R;
      if (!__all_sync(0xffffffffu, mbar_wait(&stg_full[s_], (k / R) & 1, p.err, kErrWaitFull))) break;
      if (!TF32 && k >= R &&
          !__all_sync(0xffffffffu, mbar_wait(&op_empty[s_], ((k / R) - 1) & 1, p.err, kErrWaitEmpty)))
        break;
      const unsigned char* src = staging + s_ * stage_bytes;
      unsigned char* dst = operands + s_ * stage_bytes;
      if constexpr (TF32) {
        // In place (dst == src): an elementwise map over the staged bytes.
        const int chunks = u.nload * (kSlotBytes / 16);
        for (int i = ct; i < chunks; i += kConverters) {
          float4 v = reinterpret_cast<const float4*>(src)[i];
          v.x = round_tf32(v.x * prescale);
          v.y = round_tf32(v.y * prescale);
          v.z = round_tf32(v.z * prescale);
          v.w = round_tf32(v.w * prescale);
          reinterpret_cast<float4*>(dst)[i] = v;
        }
      } else {
        // Item = (slot, row, 64-column atom, 16-byte output chunk of 8 BF16).
        unsigned char* hi = dst;
        unsigned char* lo = dst + size_t(p.nload_max) * (kSlotBytes / 2);
        const int items = u.nload * kRows * 16;
        for (int i = ct; i < items; i += kConverters) {
          const int slot = i >> 8, rem = i & 255;
          const int row = rem >> 4, atom = (rem >> 3) & 1, c = rem & 7;
          const int sw = row & 7;
          const int box = 2 * atom + (c >> 2);
          const int c0 = 2 * (c & 3);
          const unsigned char* rbase = src + slot * kSlotBytes + box * 2048 + (row >> 3) * 1024 + sw * 128;
          const float4 x0 = *reinterpret_cast<const float4*>(rbase + ((c0 ^ sw) << 4));
          const float4 x1 = *reinterpret_cast<const float4*>(rbase + (((c0 + 1) ^ sw) << 4));
          const float v[8] = {x0.x * prescale, x0.y * prescale, x0.z * prescale, x0.w * prescale,
                              x1.x * prescale, x1.y * prescale, x1.z * prescale, x1.w * prescale};
          uint4 h, l;
          split8(v, h, l);
          const int off = slot * (kSlotBytes / 2) + atom * 2048 + (row >> 3) * 1024 + sw * 128 + ((c ^ sw) << 4);
          *reinterpret_cast<uint4*>(hi + off) = h;
          *reinterpret_cast<uint4*>(lo + off) = l;
        }
      }
      fence_async_smem();  // generic-proxy writes -> visible to the tensor core
      __syncwarp();
      if (lane == 0) {
        if (!TF32) mbar_arrive(&stg_empty[s_]);
        mbar_arrive(&op_full[s_]);
      }
      const bool flush_here = (k % kStagesPerFlush) == kStagesPerFlush - 1 || k == nstages - 1;
      if (epilogue && flush_here) {
        if (!__all_sync(0xffffffffu, mbar_wait(acc_full, flushes & 1, p.err, kErrWaitFull))) break;
        tc_fence_after();
        const int m_lane = 32 * quarter + lane;  // accumulator row within the block
        const bool even = (lane & 1) == 0;
        for (int t = 0; t < u.ntask; ++t) {
          const int row_real = u.a_blk[t] * kBlock + m_lane;  // row of D
          const int m = row_real >> 1;                         // frame of the row
          for (int c0 = 0; c0 < kBlock; c0 += 32) {
            float val[32];
            tmem_ld32(tmem + (uint32_t(32 * quarter) << 16) + uint32_t(kBlock * t + c0), val);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const float o_re = __shfl_xor_sync(0xffffffffu, val[2 * i], 1);
              const float o_im = __shfl_xor_sync(0xffffffffu, val[2 * i + 1], 1);
              // Even row 2m holds (D[2m][2n], D[2m][2n+1]); its partner row 2m+1 the same columns.
              const int n = (u.b_blk[t] * kBlock + c0) / 2 + i;
              if (even && m < p.nt && n < p.nt) {
                const double re = double(val[2 * i]) + double(o_im);
                const double im = double(val[2 * i + 1]) - double(o_re);
                atomicAdd(p.upper + 2 * (size_t(m) * p.nt + n), re * factor);
                atomicAdd(p.upper + 2 * (size_t(m) * p.nt + n) + 1, im * factor);
              }
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty);
        ++flushes;
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

inline int unit_slot(const Unit& un, int blk) {
  for (int j = 0; j < un.nload; ++j)
    if (un.load[j] == blk) return j;
  return -1;
}

// Output (a, b) of a unit, staging blocks a and b if it does not yet.
inline void unit_add(Unit& un, int a, int b) {
  if (unit_slot(un, a) < 0) un.load[un.nload++] = a;
  if (unit_slot(un, b) < 0) un.load[un.nload++] = b;
  un.a_slot[un.ntask] = unit_slot(un, a);
  un.b_slot[un.ntask] = unit_slot(un, b);
  un.a_blk[un.ntask] = a;
  un.b_blk[un.ntask] = b;
  ++un.ntask;
}

// Augmenting path for diagonal block d: a unit among the first n that stages d
// and has a free output slot, possibly after moving a diagonal it holds on.
inline bool diagonal_path(int d, int nb, int n, const Unit* units, int* owner, bool* seen) {
  for (int u = 0; u < n; ++u) {
    if (seen[u] || unit_slot(units[u], d) < 0) continue;
    seen[u] = true;
    int held = 0;
    for (int e = 0; e < nb; ++e) held += owner[e] == u;
    if (units[u].ntask + held < kMaxTasks) {
      owner[d] = u;
      return true;
    }
    for (int e = 0; e < nb; ++e)
      if (owner[e] == u && diagonal_path(e, nb, n, units, owner, seen)) {
        owner[d] = u;
        return true;
      }
  }
  return false;
}

// Pack the upper 128-column blocks (b <= c) of an nb-block Gram into units of
// at most four output blocks (the 512 TMEM columns).  A CTA stages its unit's
// blocks for every row, so units are built to stage few blocks for their
// outputs: first edge-disjoint triangles {a, b, c} (three staged blocks for the
// off-diagonal outputs (a,b), (a,c), (b,c); a Steiner triple system where nb
// allows, e.g. nb = 7), then the remaining off-diagonal outputs in units of at
// most three blocks, then each diagonal output (b,b) in a unit that already
// stages b and has room (augmenting-path matching), the rest in units of up to
// three diagonals.  At most three staged blocks per unit (T = 400: 7 units of
// 4 outputs and 21 staged blocks, against 27 when rows b and nb-1-b were
// paired).  Returns the unit count, or 0.
inline int plan_units(int nb, Unit* units, int* nload_max) {
  if (nb < 1 || nb > kMaxBlocks) return 0;
  bool open[kMaxBlocks][kMaxBlocks] = {};  // off-diagonal outputs (a < b) not yet in a unit
  for (int a = 0; a < nb; ++a)
    for (int b = a + 1; b < nb; ++b) open[a][b] = true;
  int count = 0;
  auto fresh = [&]() -> Unit* {
    if (count == kMaxUnits) return nullptr;
    Unit* un = &units[count++];
    un->nload = 0;
    un->ntask = 0;
    return un;
  };
  // 1. Triangles.
  for (int a = 0; a < nb; ++a)
    for (int b = a + 1; b < nb; ++b)
      for (int c = b + 1; c < nb; ++c) {
        if (!(open[a][b] && open[a][c] && open[b][c])) continue;
        Unit* un = fresh();
        if (!un) return 0;
        unit_add(*un, a, b);
        unit_add(*un, a, c);
        unit_add(*un, b, c);
        open[a][b] = open[a][c] = open[b][c] = false;
      }
  // 2. Remaining off-diagonal outputs, up to three per unit of <= three blocks.
  for (int a = 0; a < nb; ++a)
    for (int b = a + 1; b < nb; ++b) {
      if (!open[a][b]) continue;
      Unit* un = fresh();
      if (!un) return 0;
      unit_add(*un, a, b);
      open[a][b] = false;
      for (int c = 0; c < nb && un->ntask < 3; ++c)
        for (int d = c + 1; d < nb && un->ntask < 3; ++d) {
          if (!open[c][d] || un->nload + (unit_slot(*un, c) < 0) + (unit_slot(*un, d) < 0) > 3) continue;
          unit_add(*un, c, d);
          open[c][d] = false;
        }
    }
  // 3. Diagonal outputs into units that stage their block.
  const int paired = count;
  int owner[kMaxBlocks];
  bool seen[kMaxUnits];
  for (int d = 0; d < nb; ++d) {
    owner[d] = -1;
    for (int u = 0; u < paired; ++u) seen[u] = false;
    diagonal_path(d, nb, paired, units, owner, seen);
  }
  for (int d = 0; d < nb; ++d)
    if (owner[d] >= 0) unit_add(units[owner[d]], d, d);
  // 4. Diagonal outputs left over: up to three per unit.
  Unit* rest = nullptr;
  for (int d = 0; d < nb; ++d) {
    if (owner[d] >= 0) continue;
    if (!rest || rest->ntask == 3) rest = fresh();
    if (!rest) return 0;
    unit_add(*rest, d, d);
  }
  *nload_max = 0;
  for (int u = 0; u < count; ++u)
    if (units[u].nload > *nload_max) *nload_max = units[u].nload;
  return count;
}

}  // namespace gramtc
}  // namespace rcb
