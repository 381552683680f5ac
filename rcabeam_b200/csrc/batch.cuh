// Batching form: one persistent kernel over a queue of uneven ensembles.
//
// The queue is a device table of ensembles (packed RC/CR channels, geometry,
// power output, method, frames per chunk).  Its work is flattened into items in
// queue order:
//   * OPW / XDoppler: (64-voxel tile, chunk of F frames) items of the staged
//     pipeline -- the producer warp stages the tile's windows with TMA through
//     the CTA's ring while the eight consumer warps interpolate (the same
//     device functions as the single-ensemble staged kernel);
//   * DMAS-CCF-ACF: (64-voxel tile, 32-frame chunk) items of the same staged
//     pipeline in two passes (channel-major, then angle-major), the device
//     functions of the single-ensemble DMAS kernel.
// Persistent CTAs take items from a global counter, so small and large
// ensembles share the GPU without launch gaps or tails.  XDoppler magnitudes are
// finished per tile by the CTA that completes the tile's last frame chunk, and
// the CTA that completes an ensemble's last item stamps its completion time.
// F (16, 32 or 64 frames, the producer's box width) is chosen per ensemble by
// the caller's autotuner; frames past the last whole chunk form one tail chunk
// of the next power of two >= 4 frames (its own tensor maps), as the
// single-ensemble launches split them.  A queue whose ensembles share one
// method runs a kernel compiled for that method alone (no register budget
// shared with the other methods' paths).  All staging loads are plain TMA tile
// loads.
#pragma once

#include "common.cuh"
#include "das_generic.cuh"
#include "das_staged.cuh"

namespace rcb {
namespace batch {

constexpr int kDmasLpv = 16;  // DMAS items: 32-frame chunks
constexpr int kMaxAngles = 64;

struct Ensemble {
  das::Args args;          // pointers, sizes and constants (signal unused)
  int method;              // 0 OPW, 1 XDoppler, 3 DMAS-CCF-ACF
  int lpv;                 // frames per chunk / 2: 8, 16 or 32 (staged methods)
  int lpv_tail;            // tail chunk frames / 2 (2 ... 32), 0 = no tail chunk
  int tiles, chunks;       // 64-voxel tiles x frame chunks (staged: main chunks + tail; DMAS: 32-frame chunks)
  int main_chunks;         // whole F-frame chunks
  int tma;                 // tensor maps valid (else plain staging loads)
  int pad;
  long long first_item;    // items before this ensemble
  long long tile_base;     // first per-tile counter of this ensemble
};

struct Queue {
  const Ensemble* ens;
  const CUtensorMap* maps;       // [4 n]: RC, CR main chunks, RC, CR tail chunk (64-byte aligned)
  int n;
  long long total_items;
  unsigned long long* next;      // work counter
  unsigned* done;                // [n] completed items
  unsigned* tile_done;           // per (ensemble, tile) completed chunks (XDoppler)
  unsigned long long* times;     // [n + 1]: kernel start, completion per ensemble (globaltimer ns)
  int* err;
};

// Shared-memory layout for slots of up to 2 LPV frames.
template <int LPV>
struct Smem {
  using S = das::Shape<LPV, false>;
  static constexpr size_t kData = 0;
  static constexpr size_t kTaps = size_t(das::kStages) * S::kStageBytes;
  static constexpr size_t kMeta = kTaps + size_t(das::kStages) * das::kTileVoxels * sizeof(das::StageTap);
  static constexpr size_t kFull = kMeta + 64;
  static constexpr size_t kEmpty = kFull + 8 * das::kStages;
  static constexpr size_t kVox = kEmpty + 8 * das::kStages;
  static constexpr size_t kActive = kVox + 4 * das::kTileVoxels;  // DMAS: active channels per voxel
  static constexpr size_t kItem = kActive + 4 * das::kTileVoxels;
  static constexpr size_t kAngles = kItem + 64;
  static constexpr size_t kBytes = kAngles + size_t(kMaxAngles) * 3 * sizeof(double);
};

// KIND: the queue's one method (0 OPW, 1 XDoppler, 3 DMAS), or -1 for a mixed
// queue.  TMA: 1 when every ensemble of the queue stages by TMA, 0 when none
// does, -1 to decide per ensemble (mixed queues); a kernel for one kind and one
// staging carries a single producer variant.
template <int TMA>
__device__ __forceinline__ bool use_tma(int tma) {
  if constexpr (TMA >= 0) return TMA == 1;
  return tma != 0;
}

template <int LPV, int KIND, int TMA>
__device__ __forceinline__ bool staged(const Queue& q, const das::Args& args, int method, int tma, int ei,
                                       const das::Ring& ring, const unsigned* vox, const double* angle_tab,
                                       int frame0, bool tail, uint32_t& k) {
  const int warp = threadIdx.x >> 5;
  if (warp == das::kConsumerWarps) {
    const CUtensorMap* mr = q.maps + 4 * ei + (tail ? 2 : 0);
    if constexpr (TMA != 0) {
      if (use_tma<TMA>(tma))
        return das::produce_item<LPV, false, true>(mr, mr + 1, args, vox, angle_tab, ring, frame0, k);
    }
    if constexpr (TMA != 1)
      return das::produce_item<LPV, false, false>(mr, mr + 1, args, vox, angle_tab, ring, frame0, k);
    return false;
  }
  if constexpr (KIND == 1) {
    return das::consume_item<LPV, false, das::kXdoppler>(args, vox, ring, frame0, warp, k);
  } else if constexpr (KIND == 0) {
    return das::consume_item<LPV, false, das::kOpw>(args, vox, ring, frame0, warp, k);
  } else {
    if (method == 1) return das::consume_item<LPV, false, das::kXdoppler>(args, vox, ring, frame0, warp, k);
    return das::consume_item<LPV, false, das::kOpw>(args, vox, ring, frame0, warp, k);
  }
}

template <int KIND, int TMA>
__device__ __forceinline__ bool staged_any(int lpv, const Queue& q, const das::Args& args, int method, int tma,
                                           int ei, const das::Ring& ring, const unsigned* vox,
                                           const double* angle_tab, int frame0, bool tail, uint32_t& k) {
  switch (lpv) {
    case 32: return staged<32, KIND, TMA>(q, args, method, tma, ei, ring, vox, angle_tab, frame0, tail, k);
    case 16: return staged<16, KIND, TMA>(q, args, method, tma, ei, ring, vox, angle_tab, frame0, tail, k);
    case 8: return staged<8, KIND, TMA>(q, args, method, tma, ei, ring, vox, angle_tab, frame0, tail, k);
    case 4: return staged<4, KIND, TMA>(q, args, method, tma, ei, ring, vox, angle_tab, frame0, tail, k);
    default: return staged<2, KIND, TMA>(q, args, method, tma, ei, ring, vox, angle_tab, frame0, tail, k);
  }
}

// DMAS-CCF-ACF item: 64-voxel tile x 32-frame chunk, both passes through the ring.
template <int TMA>
__device__ __forceinline__ bool staged_dmas(const Queue& q, const das::Args& args, int tma, int ei,
                                            const das::Ring& ring, const unsigned* vox, float* active,
                                            const double* angle_tab, int frame0, uint32_t& k) {
  const int warp = threadIdx.x >> 5;
  if (warp == das::kConsumerWarps) {
    const CUtensorMap* mr = q.maps + 4 * ei;
    if constexpr (TMA != 0) {
      if (use_tma<TMA>(tma))
        return das::produce_dmas_item<kDmasLpv, true>(mr, mr + 1, args, vox, angle_tab, ring, frame0, k, active);
    }
    if constexpr (TMA != 1)
      return das::produce_dmas_item<kDmasLpv, false>(mr, mr + 1, args, vox, angle_tab, ring, frame0, k, active);
    return false;
  }
  return das::consume_dmas_item<kDmasLpv>(args, vox, active, ring, frame0, warp, k);
}

// Slot width of a queue of kind KIND: 32-frame slots for DMAS alone, else 64.
template <int KIND>
__host__ __device__ constexpr int smem_lpv() { return KIND == 3 ? kDmasLpv : 32; }

// MINB resident CTAs per SM (register budget 65536 / (288 MINB)); the
// autotuner picks the variant.  KIND and TMA as for staged().
template <int MINB, int KIND, int TMA>
__global__ void __launch_bounds__(das::kThreads, MINB) run(const Queue q) {
  using Smem = batch::Smem<smem_lpv<KIND>()>;
  extern __shared__ __align__(1024) unsigned char smem[];
  const das::Ring ring{smem + Smem::kData, 0, reinterpret_cast<das::StageTap*>(smem + Smem::kTaps),
                       reinterpret_cast<int*>(smem + Smem::kMeta), reinterpret_cast<uint64_t*>(smem + Smem::kFull),
                       reinterpret_cast<uint64_t*>(smem + Smem::kEmpty)};
  unsigned* vox = reinterpret_cast<unsigned*>(smem + Smem::kVox);
  long long* item_slot = reinterpret_cast<long long*>(smem + Smem::kItem);
  int* ens_slot = reinterpret_cast<int*>(smem + Smem::kItem + 8);
  int* fail = reinterpret_cast<int*>(smem + Smem::kItem + 12);
  float* active = reinterpret_cast<float*>(smem + Smem::kActive);
  double* angle_tab = reinterpret_cast<double*>(smem + Smem::kAngles);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < das::kStages; ++s) {
      mbar_init(&ring.full[s], 32);
      mbar_init(&ring.empty[s], das::kConsumerWarps);
    }
    fence_mbar_init();
    *fail = 0;
    if (blockIdx.x == 0) atomicMin(q.times, static_cast<unsigned long long>(global_ns()));
  }
  uint32_t k = 0;  // ring position: the producer warp and each consumer warp advance it alike
  for (;;) {
    __syncthreads();  // the previous item's tables and slots are no longer read
    if (threadIdx.x == 0) {
      long long item = *fail ? q.total_items : static_cast<long long>(atomicAdd(q.next, 1ull));
      int lo = 0, hi = q.n - 1;
      if (item < q.total_items) {
        while (lo < hi) {  // last ensemble whose first item <= item
          const int mid = (lo + hi + 1) / 2;
          if (q.ens[mid].first_item <= item) lo = mid;
          else hi = mid - 1;
        }
      }
      *item_slot = item;
      *ens_slot = lo;
    }
    __syncthreads();
    const long long item = *item_slot;
    if (item >= q.total_items) break;
    const int ei = *ens_slot;
    const Ensemble& e = q.ens[ei];
    const long long local = item - e.first_item;
    const int tile = int(local / e.chunks), chunk = int(local % e.chunks);
    bool ok = true;
    const int method = e.method, tma = e.tma;
    auto item_body = [&](const das::Args& args) {
      das::load_item_tables(args, size_t(tile) * das::kTileVoxels, vox, angle_tab);
      __syncthreads();
      das::Ring r = ring;
      const int frame0 = chunk * 2 * e.lpv;
      if (KIND == 3 || (KIND < 0 && method == 3)) {
        if constexpr (KIND == 3 || KIND < 0) {
          r.slot_bytes = size_t(das::kRows) * (2 * kDmasLpv) * 8;
          ok = staged_dmas<TMA>(q, args, tma, ei, r, vox, active, angle_tab, chunk * 2 * kDmasLpv, k);
        }
      } else {
        if constexpr (KIND != 3) {
          const bool tail = chunk == e.main_chunks;
          const int lpv = tail ? e.lpv_tail : e.lpv;
          r.slot_bytes = size_t(das::kRows) * (2 * lpv) * 8;
          ok = staged_any<KIND, TMA>(lpv, q, args, method, tma, ei, r, vox, angle_tab, frame0, tail, k);
        }
      }
    };
    {
      // A private copy: the table in global memory could alias the item's
      // stores, so its fields would be reloaded inside the hot loops.
      const das::Args local = e.args;
      item_body(local);
    }
    if (!ok && lane == 0) atomicExch(fail, 1);
    __syncthreads();  // every warp's results of this item are issued
    if (threadIdx.x == 0) {
      __threadfence();
      if (KIND == 1 || (KIND < 0 && e.method == 1)) {
        // Last chunk of this tile: XDoppler magnitude |mean r conj(q)| of its voxels.
        const unsigned c = atomicAdd(q.tile_done + e.tile_base + tile, 1u) + 1;
        if (c == unsigned(e.chunks)) *item_slot = -1;  // flag for the block below
      }
      const unsigned d = atomicAdd(q.done + ei, 1u) + 1;
      if (d == unsigned(e.tiles) * unsigned(e.chunks)) q.times[1 + ei] = global_ns();
    }
    __syncthreads();
    if ((KIND == 1 || (KIND < 0 && e.method == 1)) && *item_slot == -1) {
      __threadfence();
      for (int i = threadIdx.x; i < das::kTileVoxels; i += blockDim.x) {
        const unsigned v = vox[i];
        if (v != UINT_MAX) {
          float* pd = e.args.pd + 2 * size_t(v);
          pd[0] = hypotf(__ldcg(pd), __ldcg(pd + 1));
        }
      }
    }
  }
  if (warp == das::kConsumerWarps) das::drain_ring(ring, k, q.err);
}

// Per-ensemble grid mode of the queue: a global-timer stamp after each
// ensemble's launches (start = 1: the queue's start, kept as a minimum).
__global__ void stamp(unsigned long long* t, int start) {
  if (start) atomicMin(t, static_cast<unsigned long long>(global_ns()));
  else *t = global_ns();
}

}  // namespace batch
}  // namespace rcb
