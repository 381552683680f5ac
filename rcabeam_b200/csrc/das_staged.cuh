// Frame-batched RCA delay-and-sum with TMA-staged sample windows.
//
// Work decomposition (B200, one 288-thread CTA per voxel tile x frame chunk):
//   * a tile is 64 voxels taken from a spatially compact traversal order, so
//     that for one (aperture, channel, angle) their interpolation taps fall in
//     a short window of sample rows;
//   * a producer warp walks (aperture, channel, angle) steps.  Per step it forms
//     every voxel's tap in float64 (delay, f-number aperture, window test,
//     interpolation weight, exp(+j 2 pi fd tau)), reduces the tile's row window
//     with warp reductions, writes the taps to shared memory and stages the
//     window's [16 rows x frame chunk] slab from the packed (c, a, s, t) input
//     with one cp.async.bulk.tensor load (falls back to plain loads when the
//     frame stride is not 16-byte aligned).  Windows longer than 16 rows are
//     split into overlapping sub-steps, so any voxel set is handled;
//   * eight consumer warps map lanes to (voxel, frame pair) and accumulate
//     phase * lerp(x[i0], x[i0 + 1]) in float32 registers straight from the
//     staged slab; a 4-stage mbarrier ring overlaps staging with math;
//   * the epilogue writes complex64 IQ (coalesced along frames) and adds the
//     chunk's sum |x|^2 / nt into pd.
// The reference performs the same arithmetic per unit (ensemble.cu:341-454)
// with a per-call geometry table and gathers through L1; here delays are
// formed on the fly in float64 and every gather hits shared memory.
#pragma once

#include <climits>

#include "common.cuh"

namespace rcb {
namespace das {

constexpr int kTileVoxels = 64;
constexpr int kConsumerWarps = 8;
constexpr int kThreads = (kConsumerWarps + 1) * 32;
constexpr int kRows = 16;    // sample rows per staged window
constexpr int kStages = 4;   // depth of the staging ring
constexpr int kMetaEnd = -2; // stage tag: no further steps

enum Mode : int { kOpw = 0, kXdoppler = 1, kApertures = 5 };

struct Args {
  const void* rc;
  const void* cr;
  const float* scan;
  const float* xe;
  const float* ye;
  const float* angles;
  const float* starts;
  const unsigned* order;  // traversal order (nullptr = identity)
  float* pd;
  float2* signal;
  int ns, nc, na, nt, nv;
  double c, fs, fd, fn;
  int frame_base;  // first frame of chunk 0 of this launch
  int* err;
  const double* offsets;  // [2][nc] receive-delay offsets in seconds (RC, CR), or nullptr
};

struct alignas(16) StageTap {
  int row;  // window row of the first tap, -1 = no contribution in this sub-step
  float w;
  float pr, pi;
};

template <int LPV, bool HALF>
struct Shape {
  static constexpr int kFrames = 2 * LPV;  // frames per chunk (two per lane)
  static constexpr int kElem = HALF ? 4 : 8;
  static constexpr int kRowBytes = kFrames * kElem;
  static constexpr int kStageBytes = kRows * kRowBytes;
  static constexpr size_t kOffTaps = size_t(kStages) * kStageBytes;
  static constexpr size_t kOffMeta = kOffTaps + size_t(kStages) * kTileVoxels * sizeof(StageTap);
  static constexpr size_t kOffFull = kOffMeta + 16 * ((kStages * 4 + 15) / 16);
  static constexpr size_t kOffEmpty = kOffFull + 8 * kStages;
  static constexpr size_t kOffVox = kOffEmpty + 8 * kStages;
  static constexpr size_t kOffAngles = kOffVox + 4 * kTileVoxels;
  static size_t bytes(int na) { return kOffAngles + size_t(na) * 3 * sizeof(double); }
};

template <bool HALF>
__device__ __forceinline__ float4 load_pair(const unsigned char* p) {
  if constexpr (HALF) {
    uint2 u = *reinterpret_cast<const uint2*>(p);
    float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
  } else {
    return *reinterpret_cast<const float4*>(p);
  }
}

// Shared-memory ring of one CTA: kStages slots of staged sample windows, the
// voxel taps of every slot, a slot tag and the full / empty barriers.
struct Ring {
  unsigned char* data;
  size_t slot_bytes;
  StageTap* taps;  // [kStages][kTileVoxels]
  int* meta;       // [kStages]: aperture of the slot, or kMetaEnd
  uint64_t* full;
  uint64_t* empty;
};

// Voxel ids of one 64-voxel tile and the per-angle (cos, sin, start) table.
__device__ __forceinline__ void load_item_tables(const Args& p, size_t tile0, unsigned* vox, double* angle_tab) {
  for (int i = threadIdx.x; i < kTileVoxels; i += blockDim.x) {
    size_t q = tile0 + i;
    vox[i] = q < size_t(p.nv) ? (p.order ? p.order[q] : unsigned(q)) : UINT_MAX;
  }
  for (int a = threadIdx.x; a < p.na; a += blockDim.x) {
    double th = double(p.angles[a]);
    angle_tab[3 * a] = cos(th);
    angle_tab[3 * a + 1] = sin(th);
    angle_tab[3 * a + 2] = double(p.starts[a]);
  }
}

// Producer warp of one (tile, frame chunk): stages every (aperture, channel,
// angle) window, then a kMetaEnd slot.  k is the ring position (in/out).
template <int LPV, bool HALF, bool TMA>
__device__ bool produce_item(const CUtensorMap* map_rc, const CUtensorMap* map_cr, const Args& p,
                             const unsigned* vox, const double* angle_tab, const Ring& ring, int frame0,
                             uint32_t& k) {
  using S = Shape<LPV, HALF>;
  const int lane = threadIdx.x & 31;
  double px[2], pz[2], py[2];
  bool pv[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    unsigned v = vox[lane + 32 * j];
    pv[j] = v != UINT_MAX;
    size_t b = pv[j] ? 3 * size_t(v) : 0;
    px[j] = pv[j] ? double(p.scan[b]) : 0.0;
    pz[j] = pv[j] ? double(p.scan[b + 1]) : 0.0;
    py[j] = pv[j] ? double(p.scan[b + 2]) : 0.0;
  }
  bool ok = true;
  for (int config = 0; config < 2 && ok; ++config) {
    const float* el = config ? p.ye : p.xe;
    const CUtensorMap* map = config ? map_cr : map_rc;
    const unsigned char* gsrc = static_cast<const unsigned char*>(config ? p.cr : p.rc);
    for (int ch = 0; ch < p.nc && ok; ++ch) {
      double e = double(el[ch]);
      double trx[2];
      bool act[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        trx[j] = receive_delay(config ? py[j] : px[j], pz[j], e, p.c, p.fn, &act[j]);
        if (p.offsets) trx[j] = __dadd_rn(trx[j], p.offsets[config * p.nc + ch]);
        act[j] = act[j] && pv[j];
      }
      for (int a = 0; a < p.na && ok; ++a) {
        const double cs = angle_tab[3 * a], sn = angle_tab[3 * a + 1], st = angle_tab[3 * a + 2];
        Tap t[2];
        int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          double ttx = transmit_delay(config ? px[j] : py[j], pz[j], cs, sn, p.c);
          t[j] = make_tap(__dadd_rn(ttx, trx[j]), st, p.fs, p.fd, p.ns, act[j]);
          if (t[j].i0 >= 0) {
            lo = min(lo, t[j].i0);
            hi = max(hi, t[j].i0);
          }
        }
        lo = __reduce_min_sync(0xffffffffu, lo);
        hi = __reduce_max_sync(0xffffffffu, hi);
        if (lo == INT_MAX) continue;  // no voxel of the tile sees this slab
        const int slab = ch * p.na + a;
        for (int base = lo; base <= hi; base += kRows - 1) {
          const int s = k % kStages;
          ok = __all_sync(0xffffffffu, mbar_wait(&ring.empty[s], ((k / kStages) & 1) ^ 1, p.err, kErrWaitEmpty));
          if (!ok) break;
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            int r = t[j].i0 - base;
            bool in = t[j].i0 >= 0 && r >= 0 && r < kRows - 1;
            StageTap q;
            q.row = in ? r : -1;
            q.w = t[j].w;
            q.pr = t[j].phase.x;
            q.pi = t[j].phase.y;
            ring.taps[s * kTileVoxels + lane + 32 * j] = q;
          }
          if (lane == 0) ring.meta[s] = config;
          unsigned char* dst = ring.data + size_t(s) * ring.slot_bytes;
          if constexpr (TMA) {
            __syncwarp();
            if (lane == 0) {
              mbar_arrive_expect_tx(&ring.full[s], S::kStageBytes);
              tma_load_3d(dst, map, &ring.full[s], frame0, base, slab);
            } else {
              mbar_arrive(&ring.full[s]);
            }
          } else {
            // Plain staging: zero outside the slab, like the TMA out-of-bounds fill.
            const size_t slab_off = size_t(slab) * p.ns;
            for (int i = lane; i < kRows * S::kFrames; i += 32) {
              int r = i / S::kFrames, f = i % S::kFrames;
              int row = base + r, frame = frame0 + f;
              bool inside = row < p.ns && frame < p.nt;
              size_t g = ((slab_off + size_t(inside ? row : 0)) * p.nt + size_t(inside ? frame : 0)) * S::kElem;
              if constexpr (HALF) {
                unsigned v = inside ? *reinterpret_cast<const unsigned*>(gsrc + g) : 0u;
                *reinterpret_cast<unsigned*>(dst + size_t(i) * 4) = v;
              } else {
                float2 v = inside ? *reinterpret_cast<const float2*>(gsrc + g) : make_float2(0.f, 0.f);
                *reinterpret_cast<float2*>(dst + size_t(i) * 8) = v;
              }
            }
            __syncwarp();
            mbar_arrive(&ring.full[s]);
          }
          ++k;
        }
      }
    }
  }
  if (ok) {
    const int s = k % kStages;
    ok = __all_sync(0xffffffffu, mbar_wait(&ring.empty[s], ((k / kStages) & 1) ^ 1, p.err, kErrWaitEmpty));
    if (ok) {
      if (lane == 0) ring.meta[s] = kMetaEnd;
      __syncwarp();
      mbar_arrive(&ring.full[s]);
      ++k;
    }
  }
  return ok;
}

// Every copy the producer issued has landed (before the warp may leave).
__device__ __forceinline__ void drain_ring(const Ring& ring, uint32_t k, int* err) {
  for (uint32_t u = k > kStages ? k - kStages : 0; u < k; ++u)
    mbar_wait(&ring.full[u % kStages], (u / kStages) & 1, err, kErrWaitDrain);
}

// Consumer warps (warp index cw in [0, kConsumerWarps)) of one (tile, frame
// chunk): accumulate until the kMetaEnd slot, then write IQ and power.
template <int LPV, bool HALF, int MODE>
__device__ bool consume_item(const Args& p, const unsigned* vox, const Ring& ring, int frame0, int cw, uint32_t& k) {
  using S = Shape<LPV, HALF>;
  constexpr bool kTwo = MODE != kOpw;
  const int lane = threadIdx.x & 31;
  constexpr int kVpi = 32 / LPV;  // voxels per warp instruction
  constexpr int kJ = (kTileVoxels + kConsumerWarps * kVpi - 1) / (kConsumerWarps * kVpi);
  const int vs = lane / LPV;
  const int pl = lane % LPV;
  float2 acc0[kJ][2], acc1[kJ][2];
#pragma unroll
  for (int j = 0; j < kJ; ++j) {
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      acc0[j][f] = make_float2(0.f, 0.f);
      acc1[j][f] = make_float2(0.f, 0.f);
    }
  }
  bool ok = true;
  for (;; ++k) {
    const int s = k % kStages;
    ok = __all_sync(0xffffffffu, mbar_wait(&ring.full[s], (k / kStages) & 1, p.err, kErrWaitFull));
    if (!ok) break;
    const int m = ring.meta[s];
    if (m == kMetaEnd) {
      // The end slot is consumed too (released so the ring position stays shared).
      __syncwarp();
      if (lane == 0) mbar_arrive(&ring.empty[s]);
      ++k;
      break;
    }
    const unsigned char* data = ring.data + size_t(s) * ring.slot_bytes + pl * 2 * S::kElem;
    const float4* tp = reinterpret_cast<const float4*>(ring.taps + s * kTileVoxels);
#pragma unroll
    for (int j = 0; j < kJ; ++j) {
      const int slot = (j * kConsumerWarps + cw) * kVpi + vs;
      if (slot < kTileVoxels) {
        float4 q = tp[slot];
        int row = __float_as_int(q.x);
        if (row >= 0) {
          const unsigned char* src = data + row * S::kRowBytes;
          float4 a = load_pair<HALF>(src);
          float4 b = load_pair<HALF>(src + S::kRowBytes);
          const float w = q.y;
          const float2 ph = make_float2(q.z, q.w);
          float2 v0 = make_float2(fmaf(w, b.x - a.x, a.x), fmaf(w, b.y - a.y, a.y));
          float2 v1 = make_float2(fmaf(w, b.z - a.z, a.z), fmaf(w, b.w - a.w, a.w));
          if (kTwo && m == 1) {
            acc1[j][0] = cmac(ph, v0, acc1[j][0]);
            acc1[j][1] = cmac(ph, v1, acc1[j][1]);
          } else {
            acc0[j][0] = cmac(ph, v0, acc0[j][0]);
            acc0[j][1] = cmac(ph, v1, acc0[j][1]);
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&ring.empty[s]);
  }
  if (!ok) return false;

  const float inv_nt = 1.0f / float(p.nt);
#pragma unroll
  for (int j = 0; j < kJ; ++j) {
    const int slot = (j * kConsumerWarps + cw) * kVpi + vs;
    const unsigned v = slot < kTileVoxels ? vox[slot] : UINT_MAX;
    float pr = 0.f, pi = 0.f;
    if (v != UINT_MAX) {
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const int frame = frame0 + 2 * pl + f;
        if (frame < p.nt) {
          if constexpr (MODE == kOpw) {
            float2 val = acc0[j][f];
            if (p.signal) p.signal[size_t(v) * p.nt + frame] = val;
            pr += cabs2(val);
          } else if constexpr (MODE == kApertures) {
            p.signal[size_t(2 * size_t(v)) * p.nt + frame] = acc0[j][f];
            p.signal[size_t(2 * size_t(v) + 1) * p.nt + frame] = acc1[j][f];
          } else {
            float2 val = cmul(acc0[j][f], cconj(acc1[j][f]));
            if (p.signal) p.signal[size_t(v) * p.nt + frame] = val;
            pr += val.x;
            pi += val.y;
          }
        }
      }
    }
    if constexpr (MODE != kApertures) {
#pragma unroll
      for (int off = LPV / 2; off > 0; off >>= 1) {
        pr += __shfl_xor_sync(0xffffffffu, pr, off);
        if constexpr (MODE == kXdoppler) pi += __shfl_xor_sync(0xffffffffu, pi, off);
      }
      if (pl == 0 && v != UINT_MAX) {
        atomicAdd(p.pd + 2 * size_t(v), pr * inv_nt);
        if constexpr (MODE == kXdoppler) atomicAdd(p.pd + 2 * size_t(v) + 1, pi * inv_nt);
      }
    }
  }
  return true;
}

template <int LPV, bool HALF, int MODE, bool TMA>
__global__ void __launch_bounds__(kThreads)
    opw_staged(const __grid_constant__ CUtensorMap map_rc, const __grid_constant__ CUtensorMap map_cr, Args p) {
  using S = Shape<LPV, HALF>;
  extern __shared__ __align__(1024) unsigned char smem[];
  const Ring ring{smem, S::kStageBytes, reinterpret_cast<StageTap*>(smem + S::kOffTaps),
                  reinterpret_cast<int*>(smem + S::kOffMeta), reinterpret_cast<uint64_t*>(smem + S::kOffFull),
                  reinterpret_cast<uint64_t*>(smem + S::kOffEmpty)};
  unsigned* vox = reinterpret_cast<unsigned*>(smem + S::kOffVox);
  double* angle_tab = reinterpret_cast<double*>(smem + S::kOffAngles);
  const int warp = threadIdx.x >> 5;
  const int frame0 = p.frame_base + blockIdx.y * S::kFrames;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&ring.full[s], 32);
      mbar_init(&ring.empty[s], kConsumerWarps);
    }
    fence_mbar_init();
  }
  load_item_tables(p, size_t(blockIdx.x) * kTileVoxels, vox, angle_tab);
  __syncthreads();
  uint32_t k = 0;
  if (warp == kConsumerWarps) {
    if constexpr (TMA) {
      if ((threadIdx.x & 31) == 0) {
        prefetch_tensormap(&map_rc);
        prefetch_tensormap(&map_cr);
      }
    }
    produce_item<LPV, HALF, TMA>(&map_rc, &map_cr, p, vox, angle_tab, ring, frame0, k);
    drain_ring(ring, k, p.err);
  } else {
    consume_item<LPV, HALF, MODE>(p, vox, ring, frame0, warp, k);
  }
}

// pd[2v] = |pd[2v] + j pd[2v + 1]| (XDoppler magnitude of the mean cross product).
__global__ void finish_magnitude(float* pd, size_t nv) {
  size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v < nv) pd[2 * v] = hypotf(pd[2 * v], pd[2 * v + 1]);
}

}  // namespace das
}  // namespace rcb
