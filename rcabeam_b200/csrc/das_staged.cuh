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
  static constexpr size_t kOffActive = kOffVox + 4 * kTileVoxels;  // DMAS: active channels per voxel
  static constexpr size_t kOffAngles = kOffActive + 4 * kTileVoxels;
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

// Producer-warp state of one tile: the positions of this lane's two voxels.
struct TileVoxels {
  double x[2], z[2], y[2];
  bool valid[2];
};

__device__ __forceinline__ TileVoxels tile_voxels(const Args& p, const unsigned* vox) {
  const int lane = threadIdx.x & 31;
  TileVoxels t;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    unsigned v = vox[lane + 32 * j];
    t.valid[j] = v != UINT_MAX;
    size_t b = t.valid[j] ? 3 * size_t(v) : 0;
    t.x[j] = t.valid[j] ? double(p.scan[b]) : 0.0;
    t.z[j] = t.valid[j] ? double(p.scan[b + 1]) : 0.0;
    t.y[j] = t.valid[j] ? double(p.scan[b + 2]) : 0.0;
  }
  return t;
}

// Receive delays (and f-number activity) of this lane's voxels for one channel.
__device__ __forceinline__ void receive_of(const Args& p, const TileVoxels& t, int config, int ch, double (&trx)[2],
                                           bool (&act)[2]) {
  const double e = double((config ? p.ye : p.xe)[ch]);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    trx[j] = receive_delay(config ? t.y[j] : t.x[j], t.z[j], e, p.c, p.fn, &act[j]);
    if (p.offsets) trx[j] = __dadd_rn(trx[j], p.offsets[config * p.nc + ch]);
    act[j] = act[j] && t.valid[j];
  }
}

// Stages one (aperture, channel, angle) step: the tile's taps and its sample
// window (split into overlapping 16-row sub-windows when longer), each slot
// tagged with `tag`.  Steps no voxel of the tile sees stage nothing.
template <int LPV, bool HALF, bool TMA>
__device__ __forceinline__ bool stage_step(const CUtensorMap* map, const Args& p, const TileVoxels& t,
                                           const double* angle_tab, const Ring& ring, int frame0, uint32_t& k,
                                           int config, int ch, int a, const double (&trx)[2], const bool (&act)[2],
                                           int tag) {
  using S = Shape<LPV, HALF>;
  const int lane = threadIdx.x & 31;
  const unsigned char* gsrc = static_cast<const unsigned char*>(config ? p.cr : p.rc);
  const double cs = angle_tab[3 * a], sn = angle_tab[3 * a + 1], st = angle_tab[3 * a + 2];
  Tap tp[2];
  int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    double ttx = transmit_delay(config ? t.x[j] : t.y[j], t.z[j], cs, sn, p.c);
    tp[j] = make_tap(__dadd_rn(ttx, trx[j]), st, p.fs, p.fd, p.ns, act[j]);
    if (tp[j].i0 >= 0) {
      lo = min(lo, tp[j].i0);
      hi = max(hi, tp[j].i0);
    }
  }
  lo = __reduce_min_sync(0xffffffffu, lo);
  hi = __reduce_max_sync(0xffffffffu, hi);
  if (lo == INT_MAX) return true;  // no voxel of the tile sees this slab
  const int slab = ch * p.na + a;
  for (int base = lo; base <= hi; base += kRows - 1) {
    const int s = k % kStages;
    if (!__all_sync(0xffffffffu, mbar_wait(&ring.empty[s], ((k / kStages) & 1) ^ 1, p.err, kErrWaitEmpty)))
      return false;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      int r = tp[j].i0 - base;
      bool in = tp[j].i0 >= 0 && r >= 0 && r < kRows - 1;
      StageTap q;
      q.row = in ? r : -1;
      q.w = tp[j].w;
      q.pr = tp[j].phase.x;
      q.pi = tp[j].phase.y;
      ring.taps[s * kTileVoxels + lane + 32 * j] = q;
    }
    if (lane == 0) ring.meta[s] = tag;
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
  return true;
}

// Closes an item's slot sequence with a kMetaEnd slot.
__device__ __forceinline__ bool stage_end(const Args& p, const Ring& ring, uint32_t& k) {
  const int lane = threadIdx.x & 31;
  const int s = k % kStages;
  if (!__all_sync(0xffffffffu, mbar_wait(&ring.empty[s], ((k / kStages) & 1) ^ 1, p.err, kErrWaitEmpty)))
    return false;
  if (lane == 0) ring.meta[s] = kMetaEnd;
  __syncwarp();
  mbar_arrive(&ring.full[s]);
  ++k;
  return true;
}

// Producer warp of one (tile, frame chunk): stages every (aperture, channel,
// angle) window (slot tag = aperture), then a kMetaEnd slot.  k is the ring
// position (in/out).
template <int LPV, bool HALF, bool TMA>
__device__ bool produce_item(const CUtensorMap* map_rc, const CUtensorMap* map_cr, const Args& p,
                             const unsigned* vox, const double* angle_tab, const Ring& ring, int frame0,
                             uint32_t& k) {
  const TileVoxels t = tile_voxels(p, vox);
  bool ok = true;
  for (int config = 0; config < 2 && ok; ++config) {
    const CUtensorMap* map = config ? map_cr : map_rc;
    for (int ch = 0; ch < p.nc && ok; ++ch) {
      double trx[2];
      bool act[2];
      receive_of(p, t, config, ch, trx, act);
      for (int a = 0; a < p.na && ok; ++a)
        ok = stage_step<LPV, HALF, TMA>(map, p, t, angle_tab, ring, frame0, k, config, ch, a, trx, act, config);
    }
  }
  return ok && stage_end(p, ring, k);
}

// DMAS-CCF-ACF producer (reference ensemble.cu:143-232): pass 1 walks
// (aperture, channel, angle) with tag aperture * nc + channel (per-channel sums
// over angles), pass 2 walks (aperture, angle, channel) with tag
// 2 nc + aperture * na + angle (per-angle sums over channels).  It also writes
// each voxel's count of active receive channels (both apertures) to `active`.
template <int LPV, bool TMA>
__device__ bool produce_dmas_item(const CUtensorMap* map_rc, const CUtensorMap* map_cr, const Args& p,
                                  const unsigned* vox, const double* angle_tab, const Ring& ring, int frame0,
                                  uint32_t& k, float* active) {
  const int lane = threadIdx.x & 31;
  const TileVoxels t = tile_voxels(p, vox);
  bool ok = true;
  float count[2] = {0.f, 0.f};
  for (int config = 0; config < 2 && ok; ++config) {
    const CUtensorMap* map = config ? map_cr : map_rc;
    for (int ch = 0; ch < p.nc && ok; ++ch) {
      double trx[2];
      bool act[2];
      receive_of(p, t, config, ch, trx, act);
      count[0] += float(act[0]);
      count[1] += float(act[1]);
      for (int a = 0; a < p.na && ok; ++a)
        ok = stage_step<LPV, false, TMA>(map, p, t, angle_tab, ring, frame0, k, config, ch, a, trx, act,
                                         config * p.nc + ch);
    }
  }
  active[lane] = count[0];
  active[lane + 32] = count[1];
  for (int config = 0; config < 2 && ok; ++config) {
    const CUtensorMap* map = config ? map_cr : map_rc;
    for (int a = 0; a < p.na && ok; ++a) {
      for (int ch = 0; ch < p.nc && ok; ++ch) {
        double trx[2];
        bool act[2];
        receive_of(p, t, config, ch, trx, act);
        ok = stage_step<LPV, false, TMA>(map, p, t, angle_tab, ring, frame0, k, config, ch, a, trx, act,
                                         2 * p.nc + config * p.na + a);
      }
    }
  }
  return ok && stage_end(p, ring, k);
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

// DMAS-CCF-ACF consumer warps of one (tile, frame chunk): per voxel-frame the
// slot-tag changes close a group -- a pass-1 group adds csroot and |.| of the
// channel sum to the DMAS / CCF sums, a pass-2 group adds the angle sum and
// its energy to the ACF terms -- and the epilogue forms the power
// (reference ensemble.cu:143-232, same formula as generic::nonlinear_voxel<3>).
template <int LPV>
__device__ bool consume_dmas_item(const Args& p, const unsigned* vox, const float* active, const Ring& ring,
                                  int frame0, int cw, uint32_t& k) {
  using S = Shape<LPV, false>;
  const int lane = threadIdx.x & 31;
  constexpr int kVpi = 32 / LPV;
  constexpr int kJ = (kTileVoxels + kConsumerWarps * kVpi - 1) / (kConsumerWarps * kVpi);
  const int vs = lane / LPV;
  const int pl = lane % LPV;
  float2 acc[kJ][2], ssum[kJ][2], r[kJ][2], q[kJ][2];
  float asum[kJ][2], er[kJ][2], eq[kJ][2];
#pragma unroll
  for (int j = 0; j < kJ; ++j) {
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      acc[j][f] = ssum[j][f] = r[j][f] = q[j][f] = make_float2(0.f, 0.f);
      asum[j][f] = er[j][f] = eq[j][f] = 0.f;
    }
  }
  const int pass2 = 2 * p.nc;
  int group = -1;
  auto fold = [&]() {
    if (group < 0) return;
    const bool second = group >= pass2;
    const bool cr_ap = second ? (group - pass2) >= p.na : false;
#pragma unroll
    for (int j = 0; j < kJ; ++j) {
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const float2 v = acc[j][f];
        if (!second) {
          ssum[j][f] = cadd(ssum[j][f], csroot(v));
          asum[j][f] += hypotf(v.x, v.y);
        } else if (!cr_ap) {
          r[j][f] = cadd(r[j][f], v);
          er[j][f] += cabs2(v);
        } else {
          q[j][f] = cadd(q[j][f], v);
          eq[j][f] += cabs2(v);
        }
        acc[j][f] = make_float2(0.f, 0.f);
      }
    }
  };
  bool ok = true;
  for (;; ++k) {
    const int s = k % kStages;
    ok = __all_sync(0xffffffffu, mbar_wait(&ring.full[s], (k / kStages) & 1, p.err, kErrWaitFull));
    if (!ok) break;
    const int m = ring.meta[s];
    if (m != group) {
      fold();
      group = m;
    }
    if (m == kMetaEnd) {
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
        float4 tq = tp[slot];
        int row = __float_as_int(tq.x);
        if (row >= 0) {
          const unsigned char* src = data + row * S::kRowBytes;
          float4 a0 = load_pair<false>(src);
          float4 b0 = load_pair<false>(src + S::kRowBytes);
          const float w = tq.y;
          const float2 ph = make_float2(tq.z, tq.w);
          float2 v0 = make_float2(fmaf(w, b0.x - a0.x, a0.x), fmaf(w, b0.y - a0.y, a0.y));
          float2 v1 = make_float2(fmaf(w, b0.z - a0.z, a0.z), fmaf(w, b0.w - a0.w, a0.w));
          acc[j][0] = cmac(ph, v0, acc[j][0]);
          acc[j][1] = cmac(ph, v1, acc[j][1]);
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&ring.empty[s]);
  }
  if (!ok) return false;

  const float inv = 1.0f / float(p.na);
  const float inv_nt = 1.0f / float(p.nt);
#pragma unroll
  for (int j = 0; j < kJ; ++j) {
    const int slot = (j * kConsumerWarps + cw) * kVpi + vs;
    const unsigned v = slot < kTileVoxels ? vox[slot] : UINT_MAX;
    float total = 0.f;
    if (v != UINT_MAX) {
      const float act = active[slot];
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const int frame = frame0 + 2 * pl + f;
        if (frame < p.nt) {
          const float dm = cabs2(ssum[j][f]) - asum[j][f];
          const float wc = (act > 0.f && asum[j][f] > 0.f) ? fmaxf(dm, 0.f) / act / asum[j][f] : 0.f;
          const float nr = cabs2(r[j][f]) * inv * inv, nq = cabs2(q[j][f]) * inv * inv;
          const float var = fmaxf(er[j][f] * inv - nr, 0.f) + fmaxf(eq[j][f] * inv - nq, 0.f);
          const float num = sqrtf(nr) * sqrtf(nq), den = nr + nq + var / 2 - num;
          float pw = den > 0.f ? dm * wc * (num / den) : 0.f;
          if (!isfinite(pw)) pw = 0.f;
          if (p.signal) p.signal[size_t(v) * p.nt + frame] = make_float2(pw, 0.f);
          total += pw;
        }
      }
    }
#pragma unroll
    for (int off = LPV / 2; off > 0; off >>= 1) total += __shfl_xor_sync(0xffffffffu, total, off);
    if (pl == 0 && v != UINT_MAX) atomicAdd(p.pd + 2 * size_t(v), total * inv_nt);
  }
  return true;
}

// Single-ensemble DMAS-CCF-ACF: one CTA per (tile, frame chunk), both passes
// through one staging ring.  Three resident CTAs per SM (a 72-register budget,
// a few spills) hide the single producer warp's float64 delay work: measured
// 3.7 s against 8.7 s at one CTA per SM on a 128 x 128 x 128, 11-angle,
// 200-frame ensemble.
template <int LPV, bool TMA>
__global__ void __launch_bounds__(kThreads, 3)
    dmas_staged(const __grid_constant__ CUtensorMap map_rc, const __grid_constant__ CUtensorMap map_cr, Args p) {
  using S = Shape<LPV, false>;
  extern __shared__ __align__(1024) unsigned char smem[];
  const Ring ring{smem, S::kStageBytes, reinterpret_cast<StageTap*>(smem + S::kOffTaps),
                  reinterpret_cast<int*>(smem + S::kOffMeta), reinterpret_cast<uint64_t*>(smem + S::kOffFull),
                  reinterpret_cast<uint64_t*>(smem + S::kOffEmpty)};
  unsigned* vox = reinterpret_cast<unsigned*>(smem + S::kOffVox);
  float* active = reinterpret_cast<float*>(smem + S::kOffActive);
  double* angle_tab = reinterpret_cast<double*>(smem + S::kOffAngles);
  const int warp = threadIdx.x >> 5;
  const int frame0 = blockIdx.y * S::kFrames;
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
    produce_dmas_item<LPV, TMA>(&map_rc, &map_cr, p, vox, angle_tab, ring, frame0, k, active);
    drain_ring(ring, k, p.err);
  } else {
    consume_dmas_item<LPV>(p, vox, active, ring, frame0, warp, k);
  }
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
