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
// the caller's autotuner.  All staging loads are plain TMA tile loads.
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
  int tiles, chunks;       // staged: 64-voxel tiles x frame chunks; DMAS: voxel blocks x 128-frame blocks
  int tma;                 // tensor maps valid (else plain staging loads)
  int pad;
  long long first_item;    // items before this ensemble
  long long tile_base;     // first per-tile counter of this ensemble
};

struct Queue {
  const Ensemble* ens;
  const CUtensorMap* maps;       // [2 n]: RC, CR (64-byte aligned)
  int n;
  long long total_items;
  unsigned long long* next;      // work counter
  unsigned* done;                // [n] completed items
  unsigned* tile_done;           // per (ensemble, tile) completed chunks (XDoppler)
  unsigned long long* times;     // [n + 1]: kernel start, completion per ensemble (globaltimer ns)
  int* err;
};

struct Smem {
  static constexpr int kLpv = 32;
  using S = das::Shape<kLpv, false>;
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

template <int LPV>
__device__ __forceinline__ bool staged(const Queue& q, const Ensemble& e, int ei, const das::Ring& ring,
                                       const unsigned* vox, const double* angle_tab, int frame0, uint32_t& k) {
  const int warp = threadIdx.x >> 5;
  if (warp == das::kConsumerWarps) {
    const CUtensorMap* mr = q.maps + 2 * ei;
    if (e.tma) return das::produce_item<LPV, false, true>(mr, mr + 1, e.args, vox, angle_tab, ring, frame0, k);
    return das::produce_item<LPV, false, false>(mr, mr + 1, e.args, vox, angle_tab, ring, frame0, k);
  }
  if (e.method == 1) return das::consume_item<LPV, false, das::kXdoppler>(e.args, vox, ring, frame0, warp, k);
  return das::consume_item<LPV, false, das::kOpw>(e.args, vox, ring, frame0, warp, k);
}

// DMAS-CCF-ACF item: 64-voxel tile x 32-frame chunk, both passes through the ring.
__device__ __forceinline__ bool staged_dmas(const Queue& q, const Ensemble& e, int ei, const das::Ring& ring,
                                            const unsigned* vox, float* active, const double* angle_tab, int frame0,
                                            uint32_t& k) {
  const int warp = threadIdx.x >> 5;
  if (warp == das::kConsumerWarps) {
    const CUtensorMap* mr = q.maps + 2 * ei;
    if (e.tma)
      return das::produce_dmas_item<kDmasLpv, true>(mr, mr + 1, e.args, vox, angle_tab, ring, frame0, k, active);
    return das::produce_dmas_item<kDmasLpv, false>(mr, mr + 1, e.args, vox, angle_tab, ring, frame0, k, active);
  }
  return das::consume_dmas_item<kDmasLpv>(e.args, vox, active, ring, frame0, warp, k);
}

// MINB resident CTAs per SM (register budget 65536 / (288 MINB)); the
// autotuner picks the variant.
template <int MINB>
__global__ void __launch_bounds__(das::kThreads, MINB) run(const Queue q) {
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
    {
      das::load_item_tables(e.args, size_t(tile) * das::kTileVoxels, vox, angle_tab);
      __syncthreads();
      das::Ring r = ring;
      r.slot_bytes = size_t(das::kRows) * (2 * e.lpv) * 8;
      const int frame0 = chunk * 2 * e.lpv;
      if (e.method == 3) {
        ok = staged_dmas(q, e, ei, r, vox, active, angle_tab, frame0, k);
      } else {
        switch (e.lpv) {
          case 8: ok = staged<8>(q, e, ei, r, vox, angle_tab, frame0, k); break;
          case 16: ok = staged<16>(q, e, ei, r, vox, angle_tab, frame0, k); break;
          default: ok = staged<32>(q, e, ei, r, vox, angle_tab, frame0, k); break;
        }
      }
    }
    if (!ok && lane == 0) atomicExch(fail, 1);
    __syncthreads();  // every warp's results of this item are issued
    if (threadIdx.x == 0) {
      __threadfence();
      if (e.method == 1) {
        // Last chunk of this tile: XDoppler magnitude |mean r conj(q)| of its voxels.
        const unsigned c = atomicAdd(q.tile_done + e.tile_base + tile, 1u) + 1;
        if (c == unsigned(e.chunks)) *item_slot = -1;  // flag for the block below
      }
      const unsigned d = atomicAdd(q.done + ei, 1u) + 1;
      if (d == unsigned(e.tiles) * unsigned(e.chunks)) q.times[1 + ei] = global_ns();
    }
    __syncthreads();
    if (e.method == 1 && *item_slot == -1) {
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

}  // namespace batch
}  // namespace rcb
