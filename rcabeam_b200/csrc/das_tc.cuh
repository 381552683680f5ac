// Tensor-core (tcgen05) RCA delay-and-sum: interpolation as a banded GEMM.
//
// For one (aperture, channel, angle) step and a tile of 128 spatially compact
// voxels, every voxel's two interpolation taps fall in a window of <= 16
// sample rows (about 13 on average for the full-size workload).  Writing the
// taps of a 64-voxel group as a 128 x 16 coefficient matrix A -- row 2v holds
// Re(phase * (1 - w), phase * w) of voxel v at its window rows, row 2v + 1
// the imaginary parts -- one step of one group is
//
//     D[128, 2F] += A[128, 16] . X[16, 2F]
//
// where X is the staged window of packed channel samples with real and
// imaginary parts interleaved along the frame axis (F frames, 2F <= 256
// columns).  Lane 2v of the group's TMEM accumulator then holds P = Re(A) X
// and lane 2v + 1 holds Q = Im(A) X, and the voxel's IQ is
// (P_re - Q_im) + j (P_im + Q_re).  Both 64-voxel groups of a tile use the
// same staged window (two MMAs per product), which halves the window bytes
// per interpolated sample.  Frames run in passes of nearly equal length (at
// most 128 frames, N <= 256, multiples of 8 frames; 200 = 104 + 96), so that
// every work item costs about the same and the CTAs' walks stay together.
//
// Precision: FP16-packed channels are exact FP16 and the coefficients are
// split into FP16 hi + lo (two products, coefficients scaled by 2^10 so the lo
// halves stay normal).  Float32 channels are pre-split into BF16 hi + lo
// planes; with BF16 hi/lo coefficients each step runs three products
// (Ahi Xhi + Alo Xhi + Ahi Xlo).  Accumulation is float32 in TMEM.
//
// Roles (one CTA per SM, persistent over (tile, frame pass) work items that
// the builders take from a global counter and tag every staged slot with, so
// the MMA warp and the epilogue follow them), with S ring
// stages (the deepest of 6..2 that fits shared memory; 352 threads x 168
// registers at six stages still fit the register file):
//   warps 0..S-1  builders, one per ring stage.  A warp owns whole steps:
//               channels are dealt round robin to the warps, so each warp
//               forms the float64 receive delay and phase of its channel once
//               for the 128 voxels (four per lane) and then, per angle, the
//               taps (sample index, weight, phase by angle addition with a
//               per-tile table of transmit delays and phases), the tile's row
//               window (warp reductions) and the hi / lo coefficient pairs;
//               then claims the next ring stage from a shared counter, issues
//               the window's TMA copies (64-column x 16-row SWIZZLE_128B boxes,
//               spread over lanes) and, while they fly, writes the A rows of
//               both groups from registers (bank-conflict-free 16-byte
//               stores) before its 32 arrivals on the stage's barrier;
//   warp S      TMEM allocator; lane 0 issues tcgen05.mma and commits;
//   warps S+1.. 4 epilogue warps: tcgen05.ld of both accumulators, complex
//               combine, segment sums, IQ store and power.
// Shared-memory operands: A is K-major without swizzle (8 x 16-byte core
// matrices; LBO = 128 B between the two K cores, SBO = 256 B between 8-row
// groups); X is MN-major SWIZZLE_128B straight from TMA (8-row x 128-byte
// atoms; SBO = 1024 B between K groups, LBO = 2048 B between 64-column boxes).
#pragma once

#include <climits>

#include "common.cuh"
#include "das_staged.cuh"

namespace rcb {
namespace tc {

constexpr int kVox = 128;          // voxels per tile
constexpr int kGroupVox = 64;      // voxels per M=128 MMA block
constexpr int kRows = 16;
constexpr int kStages = 4;         // default ring depth for shared-memory estimates
constexpr int kDeepStages = 6;     // deepest ring (the launcher takes the deepest of 6..2 that fits)
constexpr int kBoxCols = 64;       // 16-bit columns per TMA box (one 128-byte swizzle atom)
constexpr int kBoxBytes = kBoxCols * 2 * kRows;  // 2048
constexpr int kMaxFrames = 128;    // frames per pass: 2 x frames columns <= 256 per group
// Warps: one builder per ring stage, then the MMA warp, then 4 epilogue warps.
__host__ __device__ constexpr int threads_for(int stages) { return (stages + 1 + 4) * 32; }
constexpr int kTmemCols = 512;     // group g accumulates in columns [256 g, 256 g + 2F)
// Builders claim ring positions from a shared counter and wait for a stage by
// mbarrier parity, which is unambiguous only while a waiter is at most one
// phase ahead: that holds when no more builders than stages hold claims.
static_assert(kStages <= kDeepStages, "the deep ring is the larger one");
constexpr int kAMatBytes = 128 * kRows * 2;  // 4096: one 128 x 16 16-bit matrix
// FP16 coefficients (|c| <= 1) are scaled by 2^10 before the hi/lo split so that
// the lo halves of small coefficients stay out of the FP16 subnormal range; the
// epilogue removes the power of two exactly.
template <bool BF16X3>
constexpr float kCoefScale = BF16X3 ? 1.0f : 1024.0f;
enum Meta : int { kStep = 0, kTileEnd = 1, kFinish = 2 };
// The tensor core's float32 accumulation rounds each update toward zero, which
// shrinks a long sum by about 1.3e-8 per update (1.1e-4 of the amplitude after
// the ~8400 updates of a full-size 3-product tile).  The MMA therefore flushes
// the accumulators every kSegSteps steps; the epilogue adds the segment sums in
// float32 round-to-nearest registers and per-CTA global scratch (kMaxCtas CTAs
// x 2 groups x 64 voxels x kMaxFrames complex), which bounds the bias to the
// updates of one segment.
constexpr int kSegSteps = 512;
constexpr int kMaxCtas = 160;
constexpr size_t kPartialPerCta = size_t(2) * kGroupVox * kMaxFrames;  // float2 per CTA
enum AccKind : int { kAccPartial = 0, kAccFinal = 1, kAccFinalEmpty = 2, kAccDone = 3 };

struct Args {
  const void* x_hi[2];  // per aperture (RC, CR): FP16 or BF16 hi planes, packed (c, a, s, 2 nt)
  const void* x_lo[2];  // BF16 lo planes (three-product mode)
  const float* scan;
  const float* xe;
  const float* ye;
  const float* angles;
  const float* starts;
  const unsigned* order;
  float* pd;
  float2* signal;
  float2* partial;  // kMaxCtas x kPartialPerCta segment sums
  unsigned long long* slot_clock;  // channel slots staged by all CTAs (phase of the herd; never reset)
  int ns, nc, na, nt, nv;
  double c, fs, fd, fn;
  int frames;      // frames of every pass but the last (multiple of 8, <= 128)
  int last_frames; // frames of the last pass (multiple of 8, <= frames)
  int chunks;      // passes per tile
  int ncols;       // 2 * frames
  int nbox;        // TMA boxes per plane of a full pass (the stage layout)
  int ntiles;
  int walk_fixed;  // 1: every item walks the channel slots from slot 0 (no timing-dependent start)
  int seg_steps;   // MMA steps between accumulator flushes (float32 accumulation length)
  unsigned* item_counter;  // next work item to take (zeroed before the launch); nullptr: CTA b takes b, b + G, ...
  int* err;
};

constexpr int kCtrlBytes = 512;  // barriers, stage tags, counters, TMEM slot

template <bool BF16X3>
struct Layout {
  static constexpr int kPlanes = BF16X3 ? 2 : 1;
  // A: [group][hi, lo] matrices; then the planes' boxes.
  __host__ __device__ static size_t stage_bytes(int nbox) {
    return 4 * kAMatBytes + size_t(kPlanes) * nbox * kBoxBytes;
  }
  // stages | control (barriers, meta, counters, TMEM slot) | angle table [na][3] double |
  // per-tile transmit delay bases [2][na] double, offsets [2][na][128] float and
  // phases [2][na][128] float2 (the caller adds up to 1 KB to align the base).
  static size_t bytes(int nbox, int na, int stages) {
    return size_t(stages) * stage_bytes(nbox) + kCtrlBytes + size_t(na) * 5 * sizeof(double) +
           size_t(na) * 2 * kVox * (sizeof(float) + sizeof(float2));
  }
};

// ------------------------------------------------------------- descriptors --
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3fffu);
  d |= uint64_t((lbo >> 4) & 0x3fffu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3fffu) << 32;
  d |= uint64_t(1) << 46;  // descriptor version for sm_100
  d |= uint64_t(layout & 7u) << 61;
  return d;
}
constexpr uint32_t kLayoutNone = 0, kLayoutSw128 = 2;

// kind::f16 instruction descriptor: F32 accumulate, A K-major, B MN-major.
__host__ __device__ constexpr uint32_t instr_desc(bool bf16, int m, int n) {
  return (1u << 4) | (uint32_t(bf16) << 7) | (uint32_t(bf16) << 10) | (0u << 15) | (1u << 16) |
         (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 lanes x 32 consecutive 32-bit columns.
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16-bit split of a float: hi = round(x), lo = round(x - hi).
template <bool BF16>
__device__ __forceinline__ void split16(float x, unsigned short& hi, unsigned short& lo) {
  if constexpr (BF16) {
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
  } else {
    __half h = __float2half_rn(x);
    __half l = __float2half_rn(x - __half2float(h));
    hi = __half_as_ushort(h);
    lo = __half_as_ushort(l);
  }
}

// Byte offset of element (row m, column k) of a K-major 128 x 16 no-swizzle operand.
__device__ __forceinline__ uint32_t a_offset(int m, int k) {
  return uint32_t((m >> 3) * 256 + (k >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2);
}

// Zero one 16-element row of A hi and A lo, then store the two taps (r >= 0).
template <bool BF16>
__device__ __forceinline__ void put_row(unsigned char* a_hi, unsigned char* a_lo, int m, int r, float c0, float c1) {
  const uint32_t o0 = a_offset(m, 0), o1 = a_offset(m, 8);
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  *reinterpret_cast<uint4*>(a_hi + o0) = zero;
  *reinterpret_cast<uint4*>(a_hi + o1) = zero;
  *reinterpret_cast<uint4*>(a_lo + o0) = zero;
  *reinterpret_cast<uint4*>(a_lo + o1) = zero;
  if (r >= 0) {
    unsigned short h0, l0, h1, l1;
    split16<BF16>(c0, h0, l0);
    split16<BF16>(c1, h1, l1);
    const uint32_t e0 = a_offset(m, r), e1 = a_offset(m, r + 1);
    *reinterpret_cast<unsigned short*>(a_hi + e0) = h0;
    *reinterpret_cast<unsigned short*>(a_lo + e0) = l0;
    *reinterpret_cast<unsigned short*>(a_hi + e1) = h1;
    *reinterpret_cast<unsigned short*>(a_lo + e1) = l1;
  }
}

// Two coefficients rounded to a packed 16-bit pair (c0 in the low half) and the
// pair of their rounding residuals, rounded again: the hi / lo split of both
// taps of one A row in two conversions.
template <bool BF16>
__device__ __forceinline__ void split_pair(float c0, float c1, uint32_t& hi, uint32_t& lo) {
  if constexpr (BF16) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(c0, c1);
    const __nv_bfloat162 l = __floats2bfloat162_rn(c0 - __low2float(h), c1 - __high2float(h));
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
  } else {
    const __half2 h = __floats2half2_rn(c0, c1);
    const __half2 l = __floats2half2_rn(c0 - __low2float(h), c1 - __high2float(h));
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
  }
}

// The eight 32-bit words of a 16-column row whose only nonzero entries are the
// packed pair v at columns r, r + 1 (r = -1: an all-zero row).
struct RowPlace {
  int word;   // word holding column r (-2 when the row is empty)
  int shift;  // 0 or 16: bit offset of column r in that word
  __device__ __forceinline__ explicit RowPlace(int r) : word(r >= 0 ? r >> 1 : -2), shift((r & 1) << 4) {}
  __device__ __forceinline__ uint32_t at(int i, uint32_t v) const {
    const uint32_t first = v << shift;                      // column r (and r + 1 when r is even)
    const uint32_t second = __funnelshift_l(v, 0u, shift);  // column r + 1 when r is odd
    return i == word ? first : (i == word + 1 ? second : 0u);
  }
};

// Writes the real (row m, m even) and imaginary (row m + 1) A rows of one voxel
// into a K-major no-swizzle 128 x 16 matrix: four 16-byte stores, (row, K core)
// pieces at offsets +0 / +16 / +128 / +144.  Lanes whose 8-row group is odd
// swap the row order of each store pair, so that every store instruction of
// the warp spreads over all 32 banks (four wavefronts for 512 bytes).
__device__ __forceinline__ void put_rows(unsigned char* a, int m, const RowPlace& pl, uint32_t re, uint32_t im) {
  const bool odd = (m >> 3) & 1;
  const uint32_t base = uint32_t((m >> 3) * 256 + (m & 7) * 16);
#pragma unroll
  for (int kc = 0; kc < 2; ++kc) {
    uint4 pr, pi;
    pr.x = pl.at(4 * kc + 0, re);
    pr.y = pl.at(4 * kc + 1, re);
    pr.z = pl.at(4 * kc + 2, re);
    pr.w = pl.at(4 * kc + 3, re);
    pi.x = pl.at(4 * kc + 0, im);
    pi.y = pl.at(4 * kc + 1, im);
    pi.z = pl.at(4 * kc + 2, im);
    pi.w = pl.at(4 * kc + 3, im);
    const uint32_t o = base + 128u * kc;
    *reinterpret_cast<uint4*>(a + o + (odd ? 16u : 0u)) = odd ? pi : pr;
    *reinterpret_cast<uint4*>(a + o + (odd ? 0u : 16u)) = odd ? pr : pi;
  }
}

// mbarrier.expect_tx without an arrival: the writing warp's 32 lanes arrive
// later, once the coefficient rows are in shared memory.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait with the already-complete case inline (no call on the fast path).
__device__ __forceinline__ bool wait_phase(uint64_t* bar, uint32_t parity, int* err, int code) {
  return mbar_test(bar, parity) || mbar_wait(bar, parity, err, code);
}

// Frames of pass `chunk`: full passes of p.frames, the last one p.last_frames
// (frames beyond nt are zero-filled by TMA and never stored).
__device__ __forceinline__ int pass_frames(const Args& p, int chunk) {
  return chunk == p.chunks - 1 ? p.last_frames : p.frames;
}
__device__ __forceinline__ int pass_boxes(int frames) { return (2 * frames + kBoxCols - 1) / kBoxCols; }

// Pass of work item `item` (CTA b takes items b, b + G, b + 2G, ...; G = gridDim.x).
// The passes of a tile are consecutive items, so with G a multiple of the pass
// count a CTA would always get the same pass -- and the long and short passes
// would split the CTAs into fast and slow halves that drift apart (losing the
// lockstep that keeps the windows L2-resident) and finish unevenly.  Rotating
// the pass by the item's round makes every CTA cycle through all passes; the
// rotation is a bijection within each tile exactly when G % chunks == 0.
__device__ __forceinline__ int item_pass(const Args& p, int item) {
  const int chunk = item % p.chunks;
  if (gridDim.x % unsigned(p.chunks) != 0) return chunk;
  return (chunk + item / int(gridDim.x)) % p.chunks;
}

// exp(+j 2 pi fd tau) with the cycle count reduced in float64.
__device__ __forceinline__ float2 demod_phase(double fd, double tau) {
  double cyc = fd * tau;
  cyc -= rint(cyc);
  float sn, cs;
  sincospif(2.0f * float(cyc), &sn, &cs);
  return make_float2(cs, sn);
}

// One builder warp per ring stage: a builder waits for its stage by mbarrier
// phase parity, which is unambiguous because no more builders than stages hold
// claims (at most 2 x STAGES positions are claimed and unconsumed).
template <bool BF16X3, int STAGES>
__global__ void __launch_bounds__(threads_for(STAGES), 1)
    opw_tc(const __grid_constant__ CUtensorMap map_rc_hi, const __grid_constant__ CUtensorMap map_cr_hi,
           const __grid_constant__ CUtensorMap map_rc_lo, const __grid_constant__ CUtensorMap map_cr_lo, Args p) {
  constexpr int kBuilders = STAGES;
  constexpr int kMmaWarp = kBuilders;
  using L = Layout<BF16X3>;
  constexpr int kPlanes = L::kPlanes;
  constexpr int kProducts = BF16X3 ? 3 : 2;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // Align the working area to 1024 bytes (SWIZZLE_128B atoms).
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const size_t stage_bytes = L::stage_bytes(p.nbox);
  unsigned char* stages = smem;
  unsigned char* ctrl = smem + STAGES * stage_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(ctrl);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_empty + 1;
  int* meta = reinterpret_cast<int*>(drain + 1);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(meta + STAGES);
  int* counter = reinterpret_cast<int*>(tmem_slot + 1);  // next ring stage to claim
  int* item_steps = counter + 1;                         // steps staged for the current item
  volatile int* acc_kind = item_steps + 1;               // AccKind of the pending flush
  int* walk_start = item_steps + 2;                      // first channel slot of the current item
  int* grab = item_steps + 3;                            // the builders' current item (taken from the counter)
  volatile int* acc_item = item_steps + 4;               // work item of the pending flush
  int* meta_item = item_steps + 5;                       // [STAGES]: work item of each staged slot
  double* angle_tab = reinterpret_cast<double*>(ctrl + kCtrlBytes);
  // Transmit delay of (aperture, angle, voxel) = tx_base[aperture, angle] (the
  // tile's first voxel, float64) + tx_off (float: within a compact tile the
  // offsets stay below a few hundred ns, so float keeps them to ~1e-14 s); the
  // halved table is what lets a sixth ring stage fit beside 3xBF16 stages.
  double* tx_base = angle_tab + 3 * p.na;                                  // [2][na]
  float* tx_off = reinterpret_cast<float*>(tx_base + 2 * p.na);            // [2][na][128]
  float2* tx_phase = reinterpret_cast<float2*>(tx_off + 2 * p.na * kVox);  // [2][na][128]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 32);  // the writing builder warp
      mbar_init(&empty[s], 1);  // tcgen05.commit (or a plain arrive for markers)
    }
    mbar_init(acc_full, 2);  // tcgen05.commit + the MMA thread's release of acc_kind
    mbar_init(acc_empty, 4);
    mbar_init(drain, 1);
    *counter = 0;
    fence_mbar_init();
  }
  for (int a = threadIdx.x; a < p.na; a += blockDim.x) {
    double th = double(p.angles[a]);
    angle_tab[3 * a] = cos(th);  // float64 transmit geometry per angle
    angle_tab[3 * a + 1] = sin(th);
    angle_tab[3 * a + 2] = double(p.starts[a]);
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int work_items = p.ntiles * p.chunks;

  if (warp < kBuilders) {
    // ----------------------------------------------------------- builders --
    if (warp == 0 && lane == 0) {
      prefetch_tensormap(&map_rc_hi);
      prefetch_tensormap(&map_cr_hi);
      if constexpr (BF16X3) {
        prefetch_tensormap(&map_rc_lo);
        prefetch_tensormap(&map_cr_lo);
      }
    }
    bool ok = true;
    int nbox = p.nbox;  // boxes per plane of the current item's pass
    uint32_t tx_bytes = uint32_t(kPlanes * nbox * kBoxBytes);
    const float sc = kCoefScale<BF16X3>;
    auto builders_sync = [] { asm volatile("bar.sync 1, %0;" ::"n"(kBuilders * 32) : "memory"); };
    // Claims the next ring stage (uniform in the warp) and waits until it is free.
    auto claim = [&](uint32_t& k) -> bool {
      uint32_t mine = 0;
      if (lane == 0) mine = uint32_t(atomicAdd(counter, 1));
      k = __shfl_sync(0xffffffffu, mine, 0);
      return __all_sync(0xffffffffu,
                        wait_phase(&empty[k % STAGES], ((k / STAGES) & 1) ^ 1, p.err, kErrWaitEmpty));
    };
    // Issues the window copies of a claimed stage before its coefficient rows
    // are written (the copy's latency overlaps the row stores); the warp's 32
    // arrivals on full[s] follow the rows.
    auto issue_window = [&](uint32_t s, unsigned char* stage, int config, int col0, int row, int slab) {
      const CUtensorMap* mh = config ? &map_cr_hi : &map_rc_hi;
      const CUtensorMap* ml = config ? &map_cr_lo : &map_rc_lo;
      if (lane == 0) mbar_expect_tx(&full[s], tx_bytes);
      __syncwarp();
      unsigned char* b0 = stage + 4 * kAMatBytes;
      if (lane < kPlanes * nbox) {
        const bool second = lane >= nbox;
        const int j = second ? lane - nbox : lane;
        tma_load_3d(b0 + (second ? p.nbox : 0) * kBoxBytes + j * kBoxBytes, second ? ml : mh, &full[s],
                    col0 + j * kBoxCols, row, slab);
      }
    };
    // Stages the window [row, row + 16) x [col0, col0 + ncols) of every plane.
    auto stage_window = [&](uint32_t s, unsigned char* stage, int config, int col0, int row, int slab) {
      const CUtensorMap* mh = config ? &map_cr_hi : &map_rc_hi;
      const CUtensorMap* ml = config ? &map_cr_lo : &map_rc_lo;
      if (lane == 0) mbar_arrive_expect_tx(&full[s], tx_bytes);
      __syncwarp();
      unsigned char* b0 = stage + 4 * kAMatBytes;
      if (lane < kPlanes * nbox) {
        const bool second = lane >= nbox;
        const int j = second ? lane - nbox : lane;
        tma_load_3d(b0 + (second ? p.nbox : 0) * kBoxBytes + j * kBoxBytes, second ? ml : mh, &full[s],
                    col0 + j * kBoxCols, row, slab);
      }
      if (lane != 0) mbar_arrive(&full[s]);
    };
    for (int next = blockIdx.x;; next += gridDim.x) {
      // The next work item: b, b + G, ... for CTA b, or, with p.item_counter,
      // the next one not yet taken by any CTA (the CTAs then stay within a
      // window of consecutive items however their items' costs differ).
      int item = next;
      if (p.item_counter) {
        builders_sync();  // every builder has read the previous item's number
        if (warp == 0 && lane == 0) *grab = int(atomicAdd(p.item_counter, 1u));
        builders_sync();
        item = *grab;
      }
      if (item >= work_items) break;
      const int tile = item / p.chunks, chunk = item_pass(p, item);
      const int col0 = 2 * chunk * p.frames;
      nbox = pass_boxes(pass_frames(p, chunk));
      tx_bytes = uint32_t(kPlanes * nbox * kBoxBytes);
      // Voxels of this lane: slots lane + 32 j (group = slot / 64).
      double px[4], pz[4], py[4];
      bool pv[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const size_t q = size_t(tile) * kVox + lane + 32 * j;
        const unsigned v = q < size_t(p.nv) ? (p.order ? p.order[q] : unsigned(q)) : UINT_MAX;
        pv[j] = v != UINT_MAX;
        const size_t b3 = pv[j] ? 3 * size_t(v) : 0;
        px[j] = pv[j] ? double(p.scan[b3]) : 0.0;
        pz[j] = pv[j] ? double(p.scan[b3 + 1]) : 0.0;
        py[j] = pv[j] ? double(p.scan[b3 + 2]) : 0.0;
      }
      // Per-tile transmit table, filled cooperatively by the builder warps.
      builders_sync();  // previous item's table reads are complete
      // The tile's first slot always holds a voxel (tiles are filled in order).
      const size_t q0 = size_t(tile) * kVox;
      const size_t r3 = 3 * size_t(p.order ? p.order[q0] : unsigned(q0));
      const double x0 = double(p.scan[r3]), z0 = double(p.scan[r3 + 1]), y0 = double(p.scan[r3 + 2]);
      for (int e = warp * 32 + lane; e < 2 * p.na * kVox; e += kBuilders * 32) {
        const int v = e % kVox, ca = e / kVox, config = ca / p.na, a = ca % p.na;
        const size_t q = size_t(tile) * kVox + v;
        const unsigned vid = q < size_t(p.nv) ? (p.order ? p.order[q] : unsigned(q)) : UINT_MAX;
        const size_t b3 = vid != UINT_MAX ? 3 * size_t(vid) : 0;
        const double x = vid != UINT_MAX ? double(p.scan[b3]) : 0.0;
        const double z = vid != UINT_MAX ? double(p.scan[b3 + 1]) : 0.0;
        const double y = vid != UINT_MAX ? double(p.scan[b3 + 2]) : 0.0;
        const double ttx = transmit_delay(config ? x : y, z, angle_tab[3 * a], angle_tab[3 * a + 1], p.c);
        const double ref = transmit_delay(config ? x0 : y0, z0, angle_tab[3 * a], angle_tab[3 * a + 1], p.c);
        tx_off[e] = float(ttx - ref);
        if (v == 0) tx_base[ca] = ref;
        tx_phase[e] = demod_phase(p.fd, ttx);
      }
      // Channel slots u = aperture * nc + channel are walked from the slot the
      // other CTAs are at (the global slot count over the grid size): static
      // item assignment lets CTAs drift apart over a long launch, and CTAs in
      // different slabs together touch more sample windows than L2 holds.
      // The walk order only changes the order of the float32 sums.
      if (warp == 0 && lane == 0)
        *walk_start = p.walk_fixed ? 0 : int((*reinterpret_cast<volatile unsigned long long*>(p.slot_clock) / gridDim.x) %
                          (2ull * unsigned(p.nc)));
      builders_sync();
      int steps = 0;
      const int slots = 2 * p.nc, u0 = *walk_start;
      for (int i = warp; i < slots; i += kBuilders) {
        const int u = (u0 + i) % slots;
        const int config = u / p.nc, ch = u - config * p.nc;
        const float* el = config ? p.ye : p.xe;
        {  // this channel's receive delays, then its angles' steps
          double trx[4];
          float2 ph_rx[4];
          bool act[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            trx[j] = receive_delay(config ? py[j] : px[j], pz[j], double(el[ch]), p.c, p.fn, &act[j]);
            act[j] = act[j] && pv[j];
            ph_rx[j] = demod_phase(p.fd, trx[j]);
          }
          for (int a = 0; a < p.na; ++a) {
            const double start = angle_tab[3 * a + 2];
            const double base_tx = tx_base[config * p.na + a];
            int i0[4];
            float w[4];
            int lo = INT_MAX, hi = -1;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int ti = (config * p.na + a) * kVox + lane + 32 * j;
              const double ttx = __dadd_rn(base_tx, double(tx_off[ti]));
              const double sample = __dmul_rn(__dadd_rn(__dadd_rn(ttx, trx[j]), -start), p.fs);
              const bool in_window = act[j] && sample >= 0.0 && sample <= double(p.ns - 1);
              const double fl = floor(sample);
              i0[j] = in_window ? int(fl) : -1;
              w[j] = float(sample - fl);
              if (i0[j] >= 0) {
                lo = min(lo, i0[j]);
                hi = max(hi, i0[j]);
              }
            }
            lo = __reduce_min_sync(0xffffffffu, lo);
            hi = __reduce_max_sync(0xffffffffu, hi);
            if (lo == INT_MAX) continue;  // no voxel of the tile sees this slab
            // Hi / lo 16-bit pairs of each voxel's real and imaginary A rows.
            uint32_t re_hi[4], re_lo[4], im_hi[4], im_lo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const float2 pt = tx_phase[(config * p.na + a) * kVox + lane + 32 * j];
              const float2 ph = make_float2(pt.x * ph_rx[j].x - pt.y * ph_rx[j].y, pt.x * ph_rx[j].y + pt.y * ph_rx[j].x);
              // Coefficients of x[i0] and x[i0 + 1]: phase * (1 - w) and phase * w (scaled).
              split_pair<BF16X3>(sc * ph.x * (1.f - w[j]), sc * ph.x * w[j], re_hi[j], re_lo[j]);
              split_pair<BF16X3>(sc * ph.y * (1.f - w[j]), sc * ph.y * w[j], im_hi[j], im_lo[j]);
            }
            const int slab = ch * p.na + a;
            for (int base = lo; base <= hi; base += kRows - 1) {
              uint32_t k = 0;
              if (ok) ok = claim(k);
              if (!ok) continue;  // failed: keep the control flow, skip the work
              const uint32_t s = k % STAGES;
              unsigned char* stage = stages + size_t(s) * stage_bytes;
              issue_window(s, stage, config, col0, base, slab);
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                const int r = i0[j] - base;
                const RowPlace pl((i0[j] >= 0 && r >= 0 && r < kRows - 1) ? r : -1);
                const int g = j >> 1;                          // slots 0-63 -> group 0, 64-127 -> group 1
                const int m = 2 * (lane + 32 * (j & 1));       // A row of the voxel within its group
                unsigned char* a_hi = stage + (2 * g) * kAMatBytes;
                put_rows(a_hi, m, pl, re_hi[j], im_hi[j]);
                put_rows(a_hi + kAMatBytes, m, pl, re_lo[j], im_lo[j]);
              }
              if (lane == 0) {
                meta[s] = kStep;
                meta_item[s] = item;
              }
              fence_async_smem();
              mbar_arrive(&full[s]);
              ++steps;
            }
          }
        }
        if (lane == 0) atomicAdd(p.slot_clock, 1ull);
      }
      // Every builder's steps of this item are staged before its markers.
      builders_sync();
      if (warp == 0 && lane == 0) *item_steps = 0;
      builders_sync();
      if (lane == 0) atomicAdd(item_steps, steps);
      builders_sync();
      if (warp == 0) {
        if (*item_steps == 0) {
          // No voxel of the tile sees any sample: one all-zero step (zero
          // coefficients; window beyond the last sample, which TMA fills with
          // zeros) so that the accumulators are still initialized.
          uint32_t k = 0;
          if (ok) ok = claim(k);
          if (ok) {
            const uint32_t s = k % STAGES;
            unsigned char* stage = stages + size_t(s) * stage_bytes;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int g = j >> 1, m = 2 * (lane + 32 * (j & 1));
              put_row<BF16X3>(stage + 2 * g * kAMatBytes, stage + (2 * g + 1) * kAMatBytes, m, -1, 0.f, 0.f);
              put_row<BF16X3>(stage + 2 * g * kAMatBytes, stage + (2 * g + 1) * kAMatBytes, m + 1, -1, 0.f, 0.f);
            }
            if (lane == 0) {
              meta[s] = kStep;
              meta_item[s] = item;
            }
            fence_async_smem();
            stage_window(s, stage, 0, col0, p.ns, 0);
          }
        }
        uint32_t k = 0;
        if (ok) ok = claim(k);
        if (ok) {
          if (lane == 0) {
            meta[k % STAGES] = kTileEnd;
            meta_item[k % STAGES] = item;
          }
          mbar_arrive(&full[k % STAGES]);
        }
      }
    }
    builders_sync();  // every builder's claims are done
    if (warp == 0) {
      uint32_t k = 0;
      if (ok) ok = claim(k);
      if (ok) {
        if (lane == 0) meta[k % STAGES] = kFinish;
        mbar_arrive(&full[k % STAGES]);
      }
      // Drain: the copies of the last stages (globally last, so no later phase
      // exists on their barriers) have landed before the builders leave.
      const uint32_t total = uint32_t(*counter);
      for (uint32_t u = total > STAGES ? total - STAGES : 0; u < total; ++u)
        mbar_wait(&full[u % STAGES], (u / STAGES) & 1, p.err, kErrWaitDrain);
    }
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------------- MMA --
    if (lane == 0) {
      // The MMA shape (N) follows the pass of the work item each staged slot
      // is tagged with; every flush hands the epilogue its item.
      int cur_item = -1;
      uint32_t idesc = 0;
      uint32_t k = 0, flushes = 0;
      bool need_empty = false;  // a flush is outstanding: the epilogue must drain TMEM first
      bool issued = false;      // MMAs issued since the last flush
      int seg = 0;              // steps in the current segment
      auto flush = [&](int kind, int item) {
        *acc_kind = kind;
        *acc_item = item;
        mma_commit(acc_full);  // arrives once the segment's MMAs have completed
        mbar_arrive(acc_full);
        ++flushes;
        need_empty = true;
        issued = false;
        seg = 0;
      };
      for (;;) {
        const int s = k % STAGES;
        if (!wait_phase(&full[s], (k / STAGES) & 1, p.err, kErrWaitFull)) break;
        const int m = meta[s];
        if (need_empty) {
          if (!mbar_wait(acc_empty, (flushes - 1) & 1, p.err, kErrWaitEmpty)) break;
          need_empty = false;
        }
        if (m == kFinish) {
          flush(kAccDone, -1);  // the epilogue has drained every flush: no further item
          break;
        }
        tc_fence_after();
        if (m == kTileEnd) {
          flush(issued ? kAccFinal : kAccFinalEmpty, meta_item[s]);
          mbar_arrive(&empty[s]);
          ++k;
          continue;
        }
        if (meta_item[s] != cur_item) {
          cur_item = meta_item[s];
          idesc = instr_desc(BF16X3, 128, 2 * pass_frames(p, item_pass(p, cur_item)));
        }
        const uint32_t st = smem_u32(stages + size_t(s) * stage_bytes);
        const uint32_t b_hi = st + 4 * kAMatBytes;
        const uint32_t b_lo = b_hi + uint32_t(p.nbox * kBoxBytes);
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          const uint32_t a_hi = st + 2 * g * kAMatBytes, a_lo = a_hi + kAMatBytes;
#pragma unroll
          for (int q = 0; q < kProducts; ++q) {
            const uint32_t a = q == 1 ? a_lo : a_hi;
            const uint32_t b = q == 2 ? b_lo : b_hi;
            mma_f16(tmem + 256u * g, smem_desc(a, 128, 256, kLayoutNone), smem_desc(b, kBoxBytes, 1024, kLayoutSw128),
                    idesc, (issued || q > 0) ? 1u : 0u);
          }
        }
        issued = true;
        mma_commit(&empty[s]);  // frees the stage once these MMAs have read it
        ++k;
        if (++seg == p.seg_steps) flush(kAccPartial, cur_item);
      }
      // Every issued MMA has completed before the warp leaves (TMEM is freed after).
      mma_commit(drain);
      mbar_wait(drain, 0, p.err, kErrWaitDrain);
    }
    __syncwarp();
  } else {
    // ----------------------------------------------------------- epilogue --
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int m = 32 * q + lane;
    const bool is_p = (m & 1) == 0;
    float2* part = p.partial + size_t(blockIdx.x) * kPartialPerCta;
    uint32_t flushes = 0;
    int prev_item = -1, nflush = 0;  // nflush: earlier flushes of the same item
    {
      for (;;) {
        if (!__all_sync(0xffffffffu, mbar_wait(acc_full, flushes & 1, p.err, kErrWaitFull))) break;
        const int kind = *acc_kind;
        if (kind == kAccDone) break;
        const int item = *acc_item;
        nflush = item == prev_item ? nflush + 1 : 0;
        prev_item = item;
        const int tile = item / p.chunks, chunk = item_pass(p, item);
        const int f0 = chunk * p.frames;
        const int frames = pass_frames(p, chunk);
        tc_fence_after();
        const bool last = kind != kAccPartial;
        for (int g = 0; g < 2; ++g) {
          const int vg = m >> 1;  // voxel within the group
          // Frame-major scratch: the even lanes of a warp touch 16 consecutive float2.
          float2* pcol = part + size_t(g) * kMaxFrames * kGroupVox + vg;
          const size_t qv = size_t(tile) * kVox + kGroupVox * g + vg;
          const unsigned v = qv < size_t(p.nv) ? (p.order ? p.order[qv] : unsigned(qv)) : UINT_MAX;
          float power = 0.f;
          // Earlier segments' sums of 16 frames, loaded one chunk ahead so that
          // their L2 latency overlaps the previous chunk's TMEM read and combine.
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
            if (kind != kAccFinalEmpty) {
              tmem_ld32(tmem + (uint32_t(32 * q) << 16) + 256u * g + uint32_t(c0), val);
            } else {
#pragma unroll
              for (int i = 0; i < 32; ++i) val[i] = 0.f;
            }
            // The partner lane holds the other half (P <-> Q) of the same voxel.
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const float other_re = __shfl_xor_sync(0xffffffffu, val[2 * i], 1);
              const float other_im = __shfl_xor_sync(0xffffffffu, val[2 * i + 1], 1);
              const int fl = (c0 >> 1) + i;  // frame within the pass
              if (is_p && fl < frames) {
                // P lane: D = (P_re - Q_im, P_im + Q_re).
                float2 acc = make_float2((val[2 * i] - other_im) * (1.0f / kCoefScale<BF16X3>) + prev[i].x,
                                         (val[2 * i + 1] + other_re) * (1.0f / kCoefScale<BF16X3>) + prev[i].y);
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
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty);
        ++flushes;
      }
    }
  }
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

}  // namespace tc
}  // namespace rcb
