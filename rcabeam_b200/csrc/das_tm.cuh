// Tensor-core RCA delay-and-sum with the coefficient operand in tensor memory.
//
// The banded-GEMM formulation of das_tc.cuh (one (aperture, channel, angle)
// step of a 128-voxel tile is D[128, 2F] += A[128, 16] . X[16, 2F] per 64-voxel
// group, three BF16 products for split float32 data, two for FP16 data), with
// the traffic of shared memory cut by about 40 %: in das_tc.cuh every step
// writes four 4 KB coefficient matrices to shared memory and the six MMAs read
// them back together with the window (about 104 KB per step against 813 clocks
// of tensor work, the whole 128 B/clk of shared-memory bandwidth).  Here the
// coefficient rows are written into tensor memory with tcgen05.st and the MMAs
// take A from there (tcgen05.mma ... [d_tmem], [a_tmem], b_desc), so shared
// memory only carries the TMA window and its MMA reads.
//
// Tensor memory (512 columns x 128 lanes of 32 bits):
//   columns [0, 2 F_max)          group 0 accumulator, F_max = 104 frames
//   columns [2 F_max, 4 F_max)    group 1 accumulator
//   columns [416 + 32 a, +32)     A stage a (a < 3): g0 hi | g0 lo | g1 hi | g1 lo,
//                                 8 columns each (K = 16 BF16/FP16 values per lane,
//                                 two per column, the even one in the low half).
// Lane m of an A stage is row m of the group's A: voxel m / 2 of the group, the
// real (even m) or imaginary (odd m) coefficient row.
//
// Roles (13 warps, one persistent CTA per SM):
//   warps 0-7   two builder warpgroups.  tcgen05.st reaches only the lane
//               quarter (warp % 4) of tensor memory, so a step is built by the
//               four warps of a warpgroup together: lane l of warp q owns rows
//               32 q + l of both groups, i.e. one voxel per group and one of its
//               two rows.  Channels are dealt to the warpgroups round robin; per
//               (channel, angle) the warps form their taps (float64 delays),
//               reduce the tile's row window across the warpgroup (named barrier),
//               warp 0 claims the next ring position and issues the window's TMA
//               copies, and every warp writes its rows into the A stage;
//   warp 8      TMEM allocator; lane 0 issues tcgen05.mma and commits;
//   warps 9-12  epilogue (as das_tc.cuh).
// Rings: X windows in shared memory (kXStages deep) and A stages in tensor
// memory (kAStages deep) share one position counter k.  A builder claims k
// before its taps are known (a slab no voxel sees becomes a skip step), waits
// for the X stage before its copies and for the A stage only before its
// tcgen05.st, so the window copies run ahead of the coefficient writes.  The
// parity waits are sound because at most kBuilderGroups + kAStages positions are
// claimed and unconsumed at any time (<= 2 kAStages, <= 2 kXStages).
#pragma once

#include "das_tc.cuh"

namespace rcb {
namespace tm {

using tc::Args;
using tc::kBoxBytes;
using tc::kBoxCols;
using tc::kGroupVox;
using tc::kRows;
using tc::kVox;

constexpr int kBuilderGroups = 2;
constexpr int kBuilderWarps = 4 * kBuilderGroups;
constexpr int kMmaWarp = kBuilderWarps;
constexpr int kThreads = (kBuilderWarps + 1 + 4) * 32;  // 416
constexpr int kXStages = 6;
constexpr int kAStages = 3;
constexpr int kMaxFrames = 104;         // frames per pass (N = 2F <= 208 columns per group)
constexpr int kAccCols = 2 * kMaxFrames;  // columns per group accumulator
constexpr int kACol0 = 2 * kAccCols;      // 416: first A stage column
constexpr int kAStageCols = 32;
constexpr int kTmemCols = 512;
static_assert(kACol0 + kAStages * kAStageCols <= kTmemCols, "tensor memory budget");
static_assert(kBuilderGroups <= kAStages, "parity waits need claimed-and-unconsumed positions <= 2 x stages");
constexpr int kSegSteps = tc::kSegSteps;
constexpr size_t kPartialPerCta = size_t(2) * kGroupVox * kMaxFrames;  // float2 per CTA
enum Meta : int { kStep = 0, kTileEnd = 1, kFinish = 2, kSkip = 3 };

template <bool BF16X3>
struct Layout {
  static constexpr int kPlanes = BF16X3 ? 2 : 1;
  __host__ __device__ static size_t stage_bytes(int nbox) { return size_t(kPlanes) * nbox * kBoxBytes; }
  // X stages | control | angle table [na][3] | tx base [2][na] | tx offsets [2][na][128] float | phases float2.
  static size_t bytes(int nbox, int na) {
    return size_t(kXStages) * stage_bytes(nbox) + 1024 + size_t(na) * 5 * sizeof(double) +
           size_t(na) * 2 * kVox * (sizeof(float) + sizeof(float2));
  }
};

__device__ __forceinline__ void mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns from registers.
__device__ __forceinline__ void tmem_st32(uint32_t addr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(addr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]),
      "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]),
      "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_count(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

template <bool BF16X3>
__global__ void __launch_bounds__(kThreads, 1)
    opw_tm(const __grid_constant__ CUtensorMap map_rc_hi, const __grid_constant__ CUtensorMap map_cr_hi,
           const __grid_constant__ CUtensorMap map_rc_lo, const __grid_constant__ CUtensorMap map_cr_lo, Args p) {
  using L = Layout<BF16X3>;
  constexpr int kPlanes = L::kPlanes;
  constexpr int kProducts = BF16X3 ? 3 : 2;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const size_t xstage_bytes = L::stage_bytes(p.nbox);
  unsigned char* xring = smem;
  unsigned char* ctrl = smem + kXStages * xstage_bytes;
  uint64_t* full_x = reinterpret_cast<uint64_t*>(ctrl);
  uint64_t* empty_x = full_x + kXStages;
  uint64_t* full_a = empty_x + kXStages;
  uint64_t* empty_a = full_a + kAStages;
  uint64_t* acc_full = empty_a + kAStages;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_empty + 1;
  int* meta = reinterpret_cast<int*>(drain + 1);          // [kXStages]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(meta + kXStages);
  int* counter = reinterpret_cast<int*>(tmem_slot + 1);   // next ring position
  int* item_steps = counter + 1;
  volatile int* acc_kind = item_steps + 1;
  int* walk_start = item_steps + 2;
  // Warpgroup exchange: [group][parity] x (4 lo, 4 hi, claim).
  int* xchg = walk_start + 1;
  double* angle_tab = reinterpret_cast<double*>(ctrl + 1024);
  double* tx_base = angle_tab + 3 * p.na;                                   // [2][na]
  float* tx_off = reinterpret_cast<float*>(tx_base + 2 * p.na);             // [2][na][128]
  float2* tx_phase = reinterpret_cast<float2*>(tx_off + 2 * p.na * kVox);   // [2][na][128]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kXStages; ++s) {
      mbar_init(&full_x[s], 1);   // warp 0 of the claiming warpgroup (with the window's bytes)
      mbar_init(&empty_x[s], 1);  // tcgen05.commit or a plain arrive
    }
    for (int s = 0; s < kAStages; ++s) {
      mbar_init(&full_a[s], 4);   // the four warps of the claiming warpgroup
      mbar_init(&empty_a[s], 1);
    }
    mbar_init(acc_full, 2);
    mbar_init(acc_empty, 4);
    mbar_init(drain, 1);
    *counter = 0;
    fence_mbar_init();
  }
  for (int a = threadIdx.x; a < p.na; a += blockDim.x) {
    const double th = double(p.angles[a]);
    angle_tab[3 * a] = cos(th);
    angle_tab[3 * a + 1] = sin(th);
    angle_tab[3 * a + 2] = double(p.starts[a]);
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int work_items = p.ntiles * p.chunks;

  if (warp < kBuilderWarps) {
    // ------------------------------------------------------------ builders --
    const int group = warp >> 2, q = warp & 3;
    const int bar_id = 2 + group;
    if (warp == 0 && lane == 0) {
      prefetch_tensormap(&map_rc_hi);
      prefetch_tensormap(&map_cr_hi);
      if constexpr (BF16X3) {
        prefetch_tensormap(&map_rc_lo);
        prefetch_tensormap(&map_cr_lo);
      }
    }
    bool ok = true;
    const float sc = tc::kCoefScale<BF16X3>;
    auto all_builders = [] { asm volatile("bar.sync 1, %0;" ::"n"(kBuilderWarps * 32) : "memory"); };
    auto group_sync = [bar_id] { asm volatile("bar.sync %0, 128;" ::"r"(bar_id) : "memory"); };
    int* gx = xchg + group * 2 * 9;
    int par = 0;
    // Lane l of warp q: rows 32 q + l of both groups -> voxel slots g * 64 + 16 q + l / 2, row part l & 1.
    const int part = lane & 1;
    const int vslot0 = 16 * q + (lane >> 1);
    for (int item = blockIdx.x; item < work_items; item += gridDim.x) {
      const int tile = item / p.chunks, chunk = tc::item_pass(p, item);
      const int col0 = 2 * chunk * p.frames;
      const int nbox = tc::pass_boxes(tc::pass_frames(p, chunk));
      const uint32_t tx_bytes = uint32_t(kPlanes * nbox * kBoxBytes);
      double px[2], pz[2], py[2];
      bool pv[2];
#pragma unroll
      for (int g = 0; g < 2; ++g) {
        const size_t qv = size_t(tile) * kVox + g * kGroupVox + vslot0;
        const unsigned v = qv < size_t(p.nv) ? (p.order ? p.order[qv] : unsigned(qv)) : UINT_MAX;
        pv[g] = v != UINT_MAX;
        const size_t b3 = pv[g] ? 3 * size_t(v) : 0;
        px[g] = pv[g] ? double(p.scan[b3]) : 0.0;
        pz[g] = pv[g] ? double(p.scan[b3 + 1]) : 0.0;
        py[g] = pv[g] ? double(p.scan[b3 + 2]) : 0.0;
      }
      all_builders();  // the previous item's table reads are complete
      const size_t q0 = size_t(tile) * kVox;
      const size_t r3 = 3 * size_t(p.order ? p.order[q0] : unsigned(q0));
      const double x0 = double(p.scan[r3]), z0 = double(p.scan[r3 + 1]), y0 = double(p.scan[r3 + 2]);
      for (int e = warp * 32 + lane; e < 2 * p.na * kVox; e += kBuilderWarps * 32) {
        const int v = e % kVox, ca = e / kVox, config = ca / p.na, a = ca % p.na;
        const size_t qv = size_t(tile) * kVox + v;
        const unsigned vid = qv < size_t(p.nv) ? (p.order ? p.order[qv] : unsigned(qv)) : UINT_MAX;
        const size_t b3 = vid != UINT_MAX ? 3 * size_t(vid) : 0;
        const double x = vid != UINT_MAX ? double(p.scan[b3]) : 0.0;
        const double z = vid != UINT_MAX ? double(p.scan[b3 + 1]) : 0.0;
        const double y = vid != UINT_MAX ? double(p.scan[b3 + 2]) : 0.0;
        const double ttx = transmit_delay(config ? x : y, z, angle_tab[3 * a], angle_tab[3 * a + 1], p.c);
        const double ref = transmit_delay(config ? x0 : y0, z0, angle_tab[3 * a], angle_tab[3 * a + 1], p.c);
        tx_off[e] = float(ttx - ref);
        if (v == 0) tx_base[ca] = ref;
        tx_phase[e] = tc::demod_phase(p.fd, ttx);
      }
      if (warp == 0 && lane == 0)
        *walk_start = p.walk_fixed ? 0
                                   : int((*reinterpret_cast<volatile unsigned long long*>(p.slot_clock) / gridDim.x) %
                                         (2ull * unsigned(p.nc)));
      all_builders();
      int steps = 0;
      const int slots = 2 * p.nc, u0 = *walk_start;
      for (int i = group; i < slots; i += kBuilderGroups) {
        const int u = (u0 + i) % slots;
        const int config = u / p.nc, ch = u - config * p.nc;
        const float* el = config ? p.ye : p.xe;
        double trx[2];
        float2 ph_rx[2];
        bool act[2];
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          trx[g] = receive_delay(config ? py[g] : px[g], pz[g], double(el[ch]), p.c, p.fn, &act[g]);
          act[g] = act[g] && pv[g];
          ph_rx[g] = tc::demod_phase(p.fd, trx[g]);
        }
        for (int a = 0; a < p.na; ++a) {
          // Ring position of this slab's first window, claimed before the taps are known.
          int k = 0;
          if (q == 0 && lane == 0) k = ok ? atomicAdd(counter, 1) : 0;
          const double start = angle_tab[3 * a + 2];
          const double base_tx = tx_base[config * p.na + a];
          int i0[2];
          float w[2];
          int lo = INT_MAX, hi = -1;
#pragma unroll
          for (int g = 0; g < 2; ++g) {
            const int ti = (config * p.na + a) * kVox + g * kGroupVox + vslot0;
            const double ttx = __dadd_rn(base_tx, double(tx_off[ti]));
            const double sample = __dmul_rn(__dadd_rn(__dadd_rn(ttx, trx[g]), -start), p.fs);
            const bool in_window = act[g] && sample >= 0.0 && sample <= double(p.ns - 1);
            const double fl = floor(sample);
            i0[g] = in_window ? int(fl) : -1;
            w[g] = float(sample - fl);
            if (i0[g] >= 0) {
              lo = min(lo, i0[g]);
              hi = max(hi, i0[g]);
            }
          }
          lo = __reduce_min_sync(0xffffffffu, lo);
          hi = __reduce_max_sync(0xffffffffu, hi);
          int* slot = gx + par * 9;
          if (lane == 0) {
            slot[q] = lo;
            slot[4 + q] = hi;
            if (q == 0) slot[8] = k;
          }
          group_sync();
          lo = min(min(slot[0], slot[1]), min(slot[2], slot[3]));
          hi = max(max(slot[4], slot[5]), max(slot[6], slot[7]));
          k = slot[8];
          par ^= 1;
          if (lo == INT_MAX) {
            // No voxel of the tile sees this slab: the claimed position becomes a skip step.
            if (q == 0 && lane == 0 && ok) {
              ok = tc::wait_phase(&empty_x[k % kXStages], ((k / kXStages) & 1) ^ 1, p.err, kErrWaitEmpty);
              if (ok) {
                meta[k % kXStages] = kSkip;
                mbar_arrive(&full_x[k % kXStages]);
                ok = tc::wait_phase(&empty_a[k % kAStages], ((k / kAStages) & 1) ^ 1, p.err, kErrWaitEmpty);
                if (ok) mbar_arrive_count(&full_a[k % kAStages], 4);
              }
            }
            continue;
          }
          // This lane's row coefficients (its part of both voxels), hi / lo 16-bit pairs.
          uint32_t c_hi[2], c_lo[2];
#pragma unroll
          for (int g = 0; g < 2; ++g) {
            const float2 pt = tx_phase[(config * p.na + a) * kVox + g * kGroupVox + vslot0];
            const float2 ph = make_float2(pt.x * ph_rx[g].x - pt.y * ph_rx[g].y, pt.x * ph_rx[g].y + pt.y * ph_rx[g].x);
            const float cpart = part ? ph.y : ph.x;
            tc::split_pair<BF16X3>(sc * cpart * (1.f - w[g]), sc * cpart * w[g], c_hi[g], c_lo[g]);
          }
          const int slab = ch * p.na + a;
          for (int base = lo; base <= hi; base += kRows - 1) {
            if (base != lo) {
              // A further window of the same slab: claim another position.
              if (q == 0 && lane == 0) gx[par * 9 + 8] = ok ? atomicAdd(counter, 1) : 0;
              group_sync();
              k = gx[par * 9 + 8];
              par ^= 1;
            }
            const int sx = k % kXStages, sa = k % kAStages;
            if (q == 0) {
              // Window copies into the X stage.
              bool free_x = true;
              if (lane == 0 && ok) free_x = tc::wait_phase(&empty_x[sx], ((k / kXStages) & 1) ^ 1, p.err,
                                                           kErrWaitEmpty);
              free_x = __shfl_sync(0xffffffffu, free_x && ok, 0);
              if (free_x) {
                if (lane == 0) {
                  meta[sx] = kStep;
                  mbar_arrive_expect_tx(&full_x[sx], tx_bytes);
                }
                __syncwarp();
                if (lane < kPlanes * nbox) {
                  const bool second = lane >= nbox;
                  const int j = second ? lane - nbox : lane;
                  const CUtensorMap* m = config ? (second ? &map_cr_lo : &map_cr_hi)
                                                : (second ? &map_rc_lo : &map_rc_hi);
                  tma_load_3d(xring + size_t(sx) * xstage_bytes + size_t(second ? p.nbox : 0) * kBoxBytes +
                                  size_t(j) * kBoxBytes,
                              m, &full_x[sx], col0 + j * kBoxCols, base, slab);
                }
              }
              ok = ok && free_x;
            }
            // Rows of this window in registers: [g0 hi | g0 lo | g1 hi | g1 lo] x 8 words.
            uint32_t rows[32];
#pragma unroll
            for (int g = 0; g < 2; ++g) {
              const int r = i0[g] - base;
              const tc::RowPlace pl((i0[g] >= 0 && r >= 0 && r < kRows - 1) ? r : -1);
#pragma unroll
              for (int i = 0; i < 8; ++i) {
                rows[16 * g + i] = pl.at(i, c_hi[g]);
                rows[16 * g + 8 + i] = pl.at(i, c_lo[g]);
              }
            }
            bool free_a = true;
            if (lane == 0) free_a = tc::wait_phase(&empty_a[sa], ((k / kAStages) & 1) ^ 1, p.err, kErrWaitEmpty);
            free_a = __shfl_sync(0xffffffffu, free_a, 0);
            if (free_a) {
              tc::tc_fence_after();
              tmem_st32(tmem + (uint32_t(32 * q) << 16) + uint32_t(kACol0 + kAStageCols * sa), rows);
              tc::tc_fence_before();
              if (lane == 0) mbar_arrive(&full_a[sa]);
            }
            ok = ok && free_a;
            ++steps;
          }
        }
        if (q == 0 && lane == 0) atomicAdd(p.slot_clock, 1ull);
      }
      // Every builder's claims of this item precede its tile-end marker.
      all_builders();
      if (warp == 0 && lane == 0) *item_steps = 0;
      all_builders();
      if (q == 0 && lane == 0) atomicAdd(item_steps, steps);
      all_builders();
      if (warp == 0 && lane == 0 && ok) {
        const int k = atomicAdd(counter, 1);
        ok = tc::wait_phase(&empty_x[k % kXStages], ((k / kXStages) & 1) ^ 1, p.err, kErrWaitEmpty);
        if (ok) {
          meta[k % kXStages] = kTileEnd;
          mbar_arrive(&full_x[k % kXStages]);
          ok = tc::wait_phase(&empty_a[k % kAStages], ((k / kAStages) & 1) ^ 1, p.err, kErrWaitEmpty);
          if (ok) mbar_arrive_count(&full_a[k % kAStages], 4);
        }
      }
    }
    all_builders();
    if (warp == 0 && lane == 0) {
      if (ok) {
        const int k = atomicAdd(counter, 1);
        ok = tc::wait_phase(&empty_x[k % kXStages], ((k / kXStages) & 1) ^ 1, p.err, kErrWaitEmpty);
        if (ok) {
          meta[k % kXStages] = kFinish;
          mbar_arrive(&full_x[k % kXStages]);
        }
      }
      // Drain: the copies of the last X stages have landed before the builders leave.
      const int total = *counter;
      for (int u = total > kXStages ? total - kXStages : 0; u < total; ++u)
        mbar_wait(&full_x[u % kXStages], (u / kXStages) & 1, p.err, kErrWaitDrain);
    }
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------------- MMA --
    if (lane == 0) {
      int mma_item = blockIdx.x;
      uint32_t idesc = tc::instr_desc(BF16X3, 128, 2 * tc::pass_frames(p, tc::item_pass(p, mma_item)));
      uint32_t flushes = 0;
      bool need_empty = false, issued = false;
      int seg = 0;
      auto flush = [&](int kind) {
        *acc_kind = kind;
        tc::mma_commit(acc_full);
        mbar_arrive(acc_full);
        ++flushes;
        need_empty = true;
        issued = false;
        seg = 0;
      };
      for (int k = 0;; ++k) {
        const int sx = k % kXStages, sa = k % kAStages;
        if (!tc::wait_phase(&full_x[sx], (k / kXStages) & 1, p.err, kErrWaitFull)) break;
        const int m = meta[sx];
        if (m == kFinish) break;
        if (!tc::wait_phase(&full_a[sa], (k / kAStages) & 1, p.err, kErrWaitFull)) break;
        if (m == kSkip) {
          mbar_arrive(&empty_x[sx]);
          mbar_arrive(&empty_a[sa]);
          continue;
        }
        if (need_empty) {
          if (!mbar_wait(acc_empty, (flushes - 1) & 1, p.err, kErrWaitEmpty)) break;
          need_empty = false;
        }
        tc::tc_fence_after();
        if (m == kTileEnd) {
          flush(issued ? tc::kAccFinal : tc::kAccFinalEmpty);
          mbar_arrive(&empty_x[sx]);
          mbar_arrive(&empty_a[sa]);
          mma_item += gridDim.x;
          if (mma_item < work_items)
            idesc = tc::instr_desc(BF16X3, 128, 2 * tc::pass_frames(p, tc::item_pass(p, mma_item)));
          continue;
        }
        const uint32_t b_hi = smem_u32(xring + size_t(sx) * xstage_bytes);
        const uint32_t b_lo = b_hi + uint32_t(p.nbox * kBoxBytes);
        const uint32_t a_stage = tmem + uint32_t(kACol0 + kAStageCols * sa);
#pragma unroll
        for (int g = 0; g < 2; ++g) {
#pragma unroll
          for (int qp = 0; qp < kProducts; ++qp) {
            const uint32_t a = a_stage + uint32_t(16 * g + (qp == 1 ? 8 : 0));
            const uint32_t b = qp == 2 ? b_lo : b_hi;
            mma_ts(tmem + uint32_t(kAccCols * g), a, tc::smem_desc(b, kBoxBytes, 1024, tc::kLayoutSw128), idesc,
                   (issued || qp > 0) ? 1u : 0u);
          }
        }
        issued = true;
        tc::mma_commit(&empty_x[sx]);
        tc::mma_commit(&empty_a[sa]);
        if (++seg == p.seg_steps) flush(tc::kAccPartial);
      }
      tc::mma_commit(drain);
      mbar_wait(drain, 0, p.err, kErrWaitDrain);
    }
    __syncwarp();
  } else {
    // ----------------------------------------------------------- epilogue --
    const int q = warp & 3;
    const int m = 32 * q + lane;
    const bool is_p = (m & 1) == 0;
    float2* part = p.partial + size_t(blockIdx.x) * kPartialPerCta;
    uint32_t flushes = 0;
    bool fail = false;
    for (int item = blockIdx.x; item < work_items && !fail; item += gridDim.x) {
      const int tile = item / p.chunks, chunk = tc::item_pass(p, item);
      const int f0 = chunk * p.frames;
      const int frames = tc::pass_frames(p, chunk);
      for (int nflush = 0;; ++nflush) {
        if (!__all_sync(0xffffffffu, mbar_wait(acc_full, flushes & 1, p.err, kErrWaitFull))) {
          fail = true;
          break;
        }
        const int kind = *acc_kind;
        tc::tc_fence_after();
        const bool last = kind != tc::kAccPartial;
        for (int g = 0; g < 2; ++g) {
          const int vg = m >> 1;
          float2* pcol = part + size_t(g) * kMaxFrames * kGroupVox + vg;
          const size_t qv = size_t(tile) * kVox + kGroupVox * g + vg;
          const unsigned v = qv < size_t(p.nv) ? (p.order ? p.order[qv] : unsigned(qv)) : UINT_MAX;
          float power = 0.f;
          float2 prev[16], next[16];
          auto load_prev = [&](float2 (&dst)[16], int c0) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int fl = (c0 >> 1) + i;
              dst[i] = (nflush > 0 && is_p && fl < frames) ? pcol[size_t(fl) * kGroupVox] : make_float2(0.f, 0.f);
            }
          };
          load_prev(prev, 0);
          for (int c0 = 0; c0 < 2 * frames; c0 += 32) {
            float val[32];
            if (c0 + 32 < 2 * frames) load_prev(next, c0 + 32);
            if (kind != tc::kAccFinalEmpty) {
              tc::tmem_ld32(tmem + (uint32_t(32 * q) << 16) + uint32_t(kAccCols * g + c0), val);
            } else {
#pragma unroll
              for (int i = 0; i < 32; ++i) val[i] = 0.f;
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const float other_re = __shfl_xor_sync(0xffffffffu, val[2 * i], 1);
              const float other_im = __shfl_xor_sync(0xffffffffu, val[2 * i + 1], 1);
              const int fl = (c0 >> 1) + i;
              if (is_p && fl < frames) {
                float2 acc = make_float2((val[2 * i] - other_im) * (1.0f / tc::kCoefScale<BF16X3>) + prev[i].x,
                                         (val[2 * i + 1] + other_re) * (1.0f / tc::kCoefScale<BF16X3>) + prev[i].y);
                if (!last) {
                  pcol[size_t(fl) * kGroupVox] = acc;
                } else if (v != UINT_MAX && f0 + fl < p.nt) {
                  if (p.signal) p.signal[size_t(v) * p.nt + f0 + fl] = acc;
                  power += acc.x * acc.x + acc.y * acc.y;
                }
              }
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) prev[i] = next[i];
          }
          if (last && is_p && v != UINT_MAX) atomicAdd(p.pd + 2 * size_t(v), power / float(p.nt));
        }
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty);
        ++flushes;
        if (last) break;
      }
    }
  }
  __syncthreads();
  if (warp == kMmaWarp) {
    tc::tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

}  // namespace tm
}  // namespace rcb
