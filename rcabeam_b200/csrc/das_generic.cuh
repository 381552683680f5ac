// Frame-batched nonlinear beamformers that need per-angle or per-channel
// partial sums: RC-FMAS (method 2) and DMAS-CCF-ACF (method 3), plus the
// per-frame entry points of the reference's single-frame API (core.cu).
// One warp owns one voxel; lanes own frames (four register frames each), the
// float64 taps are formed once per (channel, angle) by every lane in lockstep.
// These are not on the OPW hot path; they keep the reference's method set and
// the batching form's mixed queue complete.
#pragma once

#include "common.cuh"
#include "das_staged.cuh"

namespace rcb {
namespace generic {

// One register frame per lane: these warp-per-voxel kernels are bound by the
// latency of their per-frame gathers, so resident warps matter more than the
// taps each 32-frame block re-forms (St-SW, k = 2: 205 ms at 4 frames, 97 ms at 1).
constexpr int kRegFrames = 1;
constexpr int kWarps = 4;

struct Voxel {
  double x, z, y;
};

__device__ __forceinline__ Voxel load_voxel(const float* scan, size_t v) {
  return Voxel{double(scan[3 * v]), double(scan[3 * v + 1]), double(scan[3 * v + 2])};
}

// Tap of (voxel, aperture config, channel, angle) from raw float inputs.
__device__ __forceinline__ Tap tap_of(const Voxel& q, int config, const float* el, int ch, const float* angles,
                                      const float* starts, int a, double c, double fs, double fd, double fn, int ns) {
  bool act;
  double trx = receive_delay(config ? q.y : q.x, q.z, double(el[ch]), c, fn, &act);
  double th = double(angles[a]);
  double ttx = transmit_delay(config ? q.x : q.y, q.z, cos(th), sin(th), c);
  return make_tap(__dadd_rn(ttx, trx), double(starts[a]), fs, fd, ns, act);
}

// Interpolated, rotated sample of a packed (c, a, s, t) complex64 ensemble.
__device__ __forceinline__ float2 packed_sample(const float2* iq, const Tap& t, int ch, int a, int frame, int ns,
                                                int na, int nt) {
  if (t.i0 < 0 || frame >= nt) return make_float2(0.f, 0.f);
  size_t idx = ((size_t(ch) * na + a) * ns + size_t(t.i0)) * nt + frame;
  size_t nxt = t.i0 == ns - 1 ? idx : idx + nt;
  float2 va = iq[idx], vb = iq[nxt];
  float2 val = make_float2(fmaf(t.w, vb.x - va.x, va.x), fmaf(t.w, vb.y - va.y, va.y));
  return cmul(val, t.phase);
}

// Transmit delays of a voxel for one angle (RC transmits along y, CR along x),
// formed once per angle with the float64 operations of tap_of.
struct AngleTx {
  double rc, cr, start;
};
__device__ __forceinline__ AngleTx angle_tx(const das::Args& p, const Voxel& q, int a) {
  const double th = double(p.angles[a]), cs = cos(th), sn = sin(th);
  return AngleTx{transmit_delay(q.y, q.z, cs, sn, p.c), transmit_delay(q.x, q.z, cs, sn, p.c), double(p.starts[a])};
}

// Tap of channel c0 + lane for one aperture (empty beyond nc): tap_of's float64
// operations with the angle's transmit delay precomputed (identical taps).
__device__ __forceinline__ Tap lane_tap_tx(const das::Args& p, const Voxel& q, int config, int c0, const AngleTx& tx) {
  const int ch = c0 + int(threadIdx.x & 31);
  if (ch >= p.nc) return Tap{-1, 0.f, make_float2(0.f, 0.f)};
  bool act;
  const double trx = receive_delay(config ? q.y : q.x, q.z, double((config ? p.ye : p.xe)[ch]), p.c, p.fn, &act);
  return make_tap(__dadd_rn(config ? tx.cr : tx.rc, trx), tx.start, p.fs, p.fd, p.ns, act);
}

__device__ __forceinline__ Tap shfl_tap(const Tap& t, int src) {
  Tap o;
  o.i0 = __shfl_sync(0xffffffffu, t.i0, src);
  o.w = __shfl_sync(0xffffffffu, t.w, src);
  o.phase.x = __shfl_sync(0xffffffffu, t.phase.x, src);
  o.phase.y = __shfl_sync(0xffffffffu, t.phase.y, src);
  return o;
}

// Taps of one aperture for channel `outer` (all angles, chan_major = false) or
// angle `outer` (all channels, chan_major = true), computed one per lane for
// the 32 inner indices starting at `first`; lanes past the end get an empty tap.
__device__ __forceinline__ Tap lane_tap(const das::Args& p, const Voxel& q, int config, bool chan_major, int outer,
                                        int first) {
  const int inner = first + (threadIdx.x & 31);
  const int limit = chan_major ? p.nc : p.na;
  if (inner >= limit) return Tap{-1, 0.f, make_float2(0.f, 0.f)};
  const int ch = chan_major ? inner : outer, a = chan_major ? outer : inner;
  return tap_of(q, config, config ? p.ye : p.xe, ch, p.angles, p.starts, a, p.c, p.fs, p.fd, p.fn, p.ns);
}

// One warp: voxel v (its row in scan / pd / signal), frames [128 fblock, 128 fblock + 128).
// The float64 taps of every (channel, angle) are formed once per warp, one per
// lane, and broadcast with shuffles.
template <int METHOD>
__device__ void nonlinear_voxel(const das::Args& p, size_t v, int fblock) {
  const int lane = threadIdx.x & 31;
  const int fbase = fblock * 32 * kRegFrames + lane;
  const Voxel q = load_voxel(p.scan, v);
  const float2* rc = static_cast<const float2*>(p.rc);
  const float2* cr = static_cast<const float2*>(p.cr);
  float power[kRegFrames];
  if constexpr (METHOD == 2) {
    // RC-FMAS: sum over angles of signed square roots of channel sums, RC * CR.
    float2 r[kRegFrames] = {}, s[kRegFrames] = {};
    // Each lane forms one channel's taps; the warp reads them back from shared memory.
    __shared__ __align__(16) Tap taps[kWarps][2][32];
    Tap* tap_rc = taps[threadIdx.x >> 5][0];
    Tap* tap_cr = taps[threadIdx.x >> 5][1];
    for (int a = 0; a < p.na; ++a) {
      float2 ar[kRegFrames] = {}, aq[kRegFrames] = {};
      const AngleTx tx = angle_tx(p, q, a);
      for (int c0 = 0; c0 < p.nc; c0 += 32) {
        __syncwarp();  // the previous chunk's reads are done
        tap_rc[lane] = lane_tap_tx(p, q, 0, c0, tx);
        tap_cr[lane] = lane_tap_tx(p, q, 1, c0, tx);
        __syncwarp();
        const int count = min(32, p.nc - c0);
        for (int j = 0; j < count; ++j) {
          const int ch = c0 + j;
          const Tap tr = tap_rc[j], tq = tap_cr[j];
#pragma unroll
          for (int f = 0; f < kRegFrames; ++f) {
            int frame = fbase + 32 * f;
            ar[f] = cadd(ar[f], packed_sample(rc, tr, ch, a, frame, p.ns, p.na, p.nt));
            aq[f] = cadd(aq[f], packed_sample(cr, tq, ch, a, frame, p.ns, p.na, p.nt));
          }
        }
      }
#pragma unroll
      for (int f = 0; f < kRegFrames; ++f) {
        r[f] = cadd(r[f], csroot(ar[f]));
        s[f] = cadd(s[f], csroot(aq[f]));
      }
    }
#pragma unroll
    for (int f = 0; f < kRegFrames; ++f) {
      float2 val = cmul(r[f], s[f]);
      int frame = fbase + 32 * f;
      if (frame < p.nt && p.signal) p.signal[v * p.nt + frame] = val;
      power[f] = frame < p.nt ? cabs2(val) : 0.f;
    }
  } else {
    // DMAS-CCF-ACF (reference ensemble.cu:143-232): pass 1 over channels for the
    // signed-sqrt DMAS and CCF terms, pass 2 over angles for the ACF terms.
    float2 sqrt_sum[kRegFrames] = {};
    float abs_sum[kRegFrames] = {};
    float active = 0.f;
    for (int ch = 0; ch < p.nc; ++ch) {
      float2 sr[kRegFrames] = {}, sq[kRegFrames] = {};
      bool act_r = false, act_q = false;
      for (int a0 = 0; a0 < p.na; a0 += 32) {
        const Tap lr = lane_tap(p, q, 0, false, ch, a0), lq = lane_tap(p, q, 1, false, ch, a0);
        const int count = min(32, p.na - a0);
        for (int j = 0; j < count; ++j) {
          const int a = a0 + j;
          const Tap tr = shfl_tap(lr, j), tq = shfl_tap(lq, j);
#pragma unroll
          for (int f = 0; f < kRegFrames; ++f) {
            int frame = fbase + 32 * f;
            sr[f] = cadd(sr[f], packed_sample(rc, tr, ch, a, frame, p.ns, p.na, p.nt));
            sq[f] = cadd(sq[f], packed_sample(cr, tq, ch, a, frame, p.ns, p.na, p.nt));
          }
        }
      }
      receive_delay(q.x, q.z, double(p.xe[ch]), p.c, p.fn, &act_r);
      receive_delay(q.y, q.z, double(p.ye[ch]), p.c, p.fn, &act_q);
      active += float(act_r) + float(act_q);
#pragma unroll
      for (int f = 0; f < kRegFrames; ++f) {
        sqrt_sum[f] = cadd(sqrt_sum[f], cadd(csroot(sr[f]), csroot(sq[f])));
        abs_sum[f] += hypotf(sr[f].x, sr[f].y) + hypotf(sq[f].x, sq[f].y);
      }
    }
    float2 r[kRegFrames] = {}, s[kRegFrames] = {};
    float er[kRegFrames] = {}, eq[kRegFrames] = {};
    for (int a = 0; a < p.na; ++a) {
      float2 ar[kRegFrames] = {}, aq[kRegFrames] = {};
      for (int c0 = 0; c0 < p.nc; c0 += 32) {
        const Tap lr = lane_tap(p, q, 0, true, a, c0), lq = lane_tap(p, q, 1, true, a, c0);
        const int count = min(32, p.nc - c0);
        for (int j = 0; j < count; ++j) {
          const int ch = c0 + j;
          const Tap tr = shfl_tap(lr, j), tq = shfl_tap(lq, j);
#pragma unroll
          for (int f = 0; f < kRegFrames; ++f) {
            int frame = fbase + 32 * f;
            ar[f] = cadd(ar[f], packed_sample(rc, tr, ch, a, frame, p.ns, p.na, p.nt));
            aq[f] = cadd(aq[f], packed_sample(cr, tq, ch, a, frame, p.ns, p.na, p.nt));
          }
        }
      }
#pragma unroll
      for (int f = 0; f < kRegFrames; ++f) {
        r[f] = cadd(r[f], ar[f]);
        s[f] = cadd(s[f], aq[f]);
        er[f] += cabs2(ar[f]);
        eq[f] += cabs2(aq[f]);
      }
    }
    const float inv = 1.0f / float(p.na);
#pragma unroll
    for (int f = 0; f < kRegFrames; ++f) {
      float dm = cabs2(sqrt_sum[f]) - abs_sum[f];
      float wc = (active > 0.f && abs_sum[f] > 0.f) ? fmaxf(dm, 0.f) / active / abs_sum[f] : 0.f;
      float nr = cabs2(r[f]) * inv * inv, nq = cabs2(s[f]) * inv * inv;
      float var = fmaxf(er[f] * inv - nr, 0.f) + fmaxf(eq[f] * inv - nq, 0.f);
      float num = sqrtf(nr) * sqrtf(nq), den = nr + nq + var / 2 - num;
      float pw = den > 0.f ? dm * wc * (num / den) : 0.f;
      if (!isfinite(pw)) pw = 0.f;
      int frame = fbase + 32 * f;
      if (frame < p.nt && p.signal) p.signal[v * p.nt + frame] = make_float2(pw, 0.f);
      power[f] = frame < p.nt ? pw : 0.f;
    }
  }
  float total = 0.f;
#pragma unroll
  for (int f = 0; f < kRegFrames; ++f) total += power[f];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) total += __shfl_xor_sync(0xffffffffu, total, off);
  if (lane == 0) atomicAdd(p.pd + 2 * v, total / float(p.nt));
}

template <int METHOD>
__global__ void __launch_bounds__(kWarps * 32) ensemble_nonlinear(das::Args p) {
  const size_t v = size_t(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (v >= size_t(p.nv)) return;
  nonlinear_voxel<METHOD>(p, v, blockIdx.y);
}

// ------------------------------------------------------------ St-SW --
// St-SW (method 4; reference stsw.py:10-107, ensemble.cu:457-627).  Angles of
// each aperture fall into K interleaved subsets (a % K).  Per frame: the
// subset means m and mean squared deviations v of the per-angle sums, the
// K x K series c[i][j] = m_rc[i] conj(m_cr[j]) / (|m_rc[i]|^2 + |m_cr[j]|^2 +
// (v_rc[i] + v_cr[j]) / 2 - |m_rc[i] conj(m_cr[j])|); over frames the raw
// weight |sum over (i1 < i2, j1 != j2) of sum_t c1 conj(c2) / sqrt(E1 E2)| with
// E the series energies; the power is the XDoppler |mean_t r conj(q)|.
//
// Pass 1 (one warp per voxel, lanes over frames): per-angle channel sums in
// angle-major order with the taps broadcast as for RC-FMAS, Welford updates of
// the subset statistics (no E|x|^2 - |E x|^2 cancellation), the series written
// to the caller's workspace (v K^2 + i K + j) nt + t and r conj(q) summed into
// pd[2v], pd[2v + 1].
template <int K, int RF>
__global__ void __launch_bounds__(kWarps * 32) stsw_series(das::Args p, float2* series) {
  const size_t v = size_t(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (v >= size_t(p.nv)) return;
  const int lane = threadIdx.x & 31;
  const int fbase = blockIdx.y * 32 * RF + lane;
  const Voxel q = load_voxel(p.scan, v);
  const float2* rc = static_cast<const float2*>(p.rc);
  const float2* cr = static_cast<const float2*>(p.cr);
  __shared__ __align__(16) Tap taps[kWarps][2][32];
  Tap* tap_rc = taps[threadIdx.x >> 5][0];
  Tap* tap_cr = taps[threadIdx.x >> 5][1];
  float2 r[RF] = {}, s[RF] = {};
  float2 mr[K][RF] = {}, mq[K][RF] = {};
  float vr[K][RF] = {}, vq[K][RF] = {};
  for (int a = 0; a < p.na; ++a) {
    float2 ar[RF] = {}, aq[RF] = {};
    const AngleTx tx = angle_tx(p, q, a);  // the voxel's transmit delays, once per angle
    for (int c0 = 0; c0 < p.nc; c0 += 32) {
      // Each lane forms one channel's taps; the warp then reads them back from
      // shared memory (one broadcast 16-byte load per tap instead of four shuffles).
      __syncwarp();  // the previous chunk's reads are done
      tap_rc[lane] = lane_tap_tx(p, q, 0, c0, tx);
      tap_cr[lane] = lane_tap_tx(p, q, 1, c0, tx);
      __syncwarp();
      const int count = min(32, p.nc - c0);
      for (int j = 0; j < count; ++j) {
        const int ch = c0 + j;
        const Tap tr = tap_rc[j], tq = tap_cr[j];
#pragma unroll
        for (int f = 0; f < RF; ++f) {
          const int frame = fbase + 32 * f;
          ar[f] = cadd(ar[f], packed_sample(rc, tr, ch, a, frame, p.ns, p.na, p.nt));
          aq[f] = cadd(aq[f], packed_sample(cr, tq, ch, a, frame, p.ns, p.na, p.nt));
        }
      }
    }
    // Welford update of subset a % K, whose (a / K + 1)-th angle this is.
    const int subset = a % K;
    const float inv = 1.0f / float(a / K + 1);
#pragma unroll
    for (int f = 0; f < RF; ++f) {
      r[f] = cadd(r[f], ar[f]);
      s[f] = cadd(s[f], aq[f]);
#pragma unroll
      for (int i = 0; i < K; ++i) {
        if (i != subset) continue;
        const float2 dr = make_float2(ar[f].x - mr[i][f].x, ar[f].y - mr[i][f].y);
        const float2 dq = make_float2(aq[f].x - mq[i][f].x, aq[f].y - mq[i][f].y);
        mr[i][f] = make_float2(fmaf(dr.x, inv, mr[i][f].x), fmaf(dr.y, inv, mr[i][f].y));
        mq[i][f] = make_float2(fmaf(dq.x, inv, mq[i][f].x), fmaf(dq.y, inv, mq[i][f].y));
        vr[i][f] += dr.x * (ar[f].x - mr[i][f].x) + dr.y * (ar[f].y - mr[i][f].y);
        vq[i][f] += dq.x * (aq[f].x - mq[i][f].x) + dq.y * (aq[f].y - mq[i][f].y);
      }
    }
  }
  float cross_re = 0.f, cross_im = 0.f;
#pragma unroll
  for (int f = 0; f < RF; ++f) {
    const int frame = fbase + 32 * f;
    if (frame >= p.nt) continue;
    const float2 x = cmul(r[f], cconj(s[f]));
    cross_re += x.x;
    cross_im += x.y;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      // Subset i holds the angles i, i + K, ... < na.
      const float count = float((p.na - 1 - i) / K + 1);
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const float countq = float((p.na - 1 - j) / K + 1);
        const float2 num = cmul(mr[i][f], cconj(mq[j][f]));
        const float den = cabs2(mr[i][f]) + cabs2(mq[j][f]) + (vr[i][f] / count + vq[j][f] / countq) * 0.5f -
                          hypotf(num.x, num.y);
        float2 value = den > 0.f ? make_float2(num.x / den, num.y / den) : make_float2(0.f, 0.f);
        if (!isfinite(value.x) || !isfinite(value.y)) value = make_float2(0.f, 0.f);
        series[(v * (K * K) + size_t(i * K + j)) * size_t(p.nt) + size_t(frame)] = value;
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    cross_re += __shfl_xor_sync(0xffffffffu, cross_re, off);
    cross_im += __shfl_xor_sync(0xffffffffu, cross_im, off);
  }
  if (lane == 0) {
    atomicAdd(p.pd + 2 * v, cross_re / float(p.nt));
    atomicAdd(p.pd + 2 * v + 1, cross_im / float(p.nt));
  }
}

// Pass 2 (one warp per voxel): series energies over frames, then the pair sum
// with running row / column sums of the normalized series (for row i, the
// earlier rows' total minus their column j pairs with c[i][j]), the raw weight
// |acc| and the XDoppler magnitude in pd[2v].
template <int K>
__global__ void __launch_bounds__(kWarps * 32) stsw_finish(float* pd, float* weights, const float2* series,
                                                           size_t nv, int nt) {
  const size_t v = size_t(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (v >= nv) return;
  const int lane = threadIdx.x & 31;
  const float2* base = series + v * (K * K) * size_t(nt);
  float scale[K * K];
#pragma unroll
  for (int e = 0; e < K * K; ++e) {
    float energy = 0.f;
    for (int t = lane; t < nt; t += 32) energy += cabs2(base[size_t(e) * nt + t]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) energy += __shfl_xor_sync(0xffffffffu, energy, off);
    scale[e] = energy > 0.f ? 1.0f / sqrtf(energy) : 0.f;
  }
  float2 acc = make_float2(0.f, 0.f);
  for (int t = lane; t < nt; t += 32) {
    float2 total = make_float2(0.f, 0.f), column[K] = {};
#pragma unroll
    for (int i = 0; i < K; ++i) {
      float2 row = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const float2 raw = base[size_t(i * K + j) * nt + t];
        const float2 value = make_float2(raw.x * scale[i * K + j], raw.y * scale[i * K + j]);
        const float2 earlier = make_float2(total.x - column[j].x, total.y - column[j].y);
        acc = cadd(acc, cmul(earlier, cconj(value)));
        column[j] = cadd(column[j], value);
        row = cadd(row, value);
      }
      total = cadd(total, row);
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
  }
  if (lane == 0) {
    weights[v] = hypotf(acc.x, acc.y);
    pd[2 * v] = hypotf(pd[2 * v], pd[2 * v + 1]);
  }
}

// --------------------------------------------- single-frame API (core.cu) --
// Channel layout (samples, channels, angles); one frame.
__device__ __forceinline__ float2 frame_sample(const float2* iq, const Voxel& q, const float* el, const float* angles,
                                               const float* starts, int ns, int nc, int na, int ch, int a, int config,
                                               double c, double fs, double fd, double fn) {
  Tap t = tap_of(q, config, el, ch, angles, starts, a, c, fs, fd, fn, ns);
  if (t.i0 < 0) return make_float2(0.f, 0.f);
  size_t i0 = (size_t(t.i0) * nc + ch) * na + a;
  size_t i1 = (size_t(t.i0 == ns - 1 ? t.i0 : t.i0 + 1) * nc + ch) * na + a;
  float2 va = iq[i0], vb = iq[i1];
  float2 val = make_float2(fmaf(t.w, vb.x - va.x, va.x), fmaf(t.w, vb.y - va.y, va.y));
  return cmul(val, t.phase);
}

struct FrameArgs {
  const float2* rc;
  const float2* cr;
  const float* scan;
  const float* xe;
  const float* ye;
  const float* angles;
  const float* starts;
  int ns, nc, na;
  size_t nv;
  double c, fs, fd, fn;
};

// out[v, a] = sum over channels (one aperture).
__global__ void frame_angle_sums(FrameArgs p, int config, float2* out) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= p.nv * p.na) return;
  size_t v = i / p.na;
  int a = int(i % p.na);
  Voxel q = load_voxel(p.scan, v);
  float2 acc = make_float2(0.f, 0.f);
  for (int ch = 0; ch < p.nc; ++ch)
    acc = cadd(acc, frame_sample(p.rc, q, p.xe, p.angles, p.starts, p.ns, p.nc, p.na, ch, a, config, p.c, p.fs, p.fd,
                                 p.fn));
  out[i] = acc;
}

// channel_sum[v, c] = sum over angles; n_active[v] = active channel count.
__global__ void frame_channel_sums(FrameArgs p, int config, float2* channel_sum, float* n_active) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= p.nv * p.nc) return;
  size_t v = i / p.nc;
  int ch = int(i % p.nc);
  Voxel q = load_voxel(p.scan, v);
  float2 acc = make_float2(0.f, 0.f);
  for (int a = 0; a < p.na; ++a)
    acc = cadd(acc, frame_sample(p.rc, q, p.xe, p.angles, p.starts, p.ns, p.nc, p.na, ch, a, config, p.c, p.fs, p.fd,
                                 p.fn));
  channel_sum[i] = acc;
  if (ch == 0) {
    float count = 0.f;
    for (int e = 0; e < p.nc; ++e) {
      bool act;
      receive_delay(config ? q.y : q.x, q.z, double(p.xe[e]), p.c, p.fn, &act);
      count += act ? 1.f : 0.f;
    }
    n_active[v] = count;
  }
}

enum FrameOut : int { kFrameOpw = 1, kFrameXd = 2, kFrameFmas = 4, kFrameDmas = 8 };

// Per-voxel single-frame reductions of both apertures.
__global__ void frame_reduce(FrameArgs p, int which, float* opw_out, float* xd_out, float* fmas_out,
                             float* dmas_out) {
  size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= p.nv) return;
  Voxel q = load_voxel(p.scan, v);
  float2 opw = {}, rsum = {}, qsum = {}, fr = {}, fq = {};
  float er = 0.f, eq = 0.f;
  for (int a = 0; a < p.na; ++a) {
    float2 ra = {}, qa = {};
    for (int ch = 0; ch < p.nc; ++ch) {
      ra = cadd(ra, frame_sample(p.rc, q, p.xe, p.angles, p.starts, p.ns, p.nc, p.na, ch, a, 0, p.c, p.fs, p.fd, p.fn));
      qa = cadd(qa, frame_sample(p.cr, q, p.ye, p.angles, p.starts, p.ns, p.nc, p.na, ch, a, 1, p.c, p.fs, p.fd, p.fn));
    }
    opw = cadd(opw, cadd(ra, qa));
    rsum = cadd(rsum, ra);
    qsum = cadd(qsum, qa);
    fr = cadd(fr, csroot(ra));
    fq = cadd(fq, csroot(qa));
    er += cabs2(ra);
    eq += cabs2(qa);
  }
  if (which & kFrameOpw) opw_out[v] = cabs2(opw);
  if (which & kFrameXd) {
    float2 x = cmul(rsum, cconj(qsum));
    xd_out[v] = hypotf(x.x, x.y);
  }
  if (which & kFrameFmas) fmas_out[v] = cabs2(cmul(fr, fq));
  if (which & kFrameDmas) {
    float2 sqrt_sum = {};
    float abs_sum = 0.f, active = 0.f;
    for (int ch = 0; ch < p.nc; ++ch) {
      float2 sr = {}, sq = {};
      for (int a = 0; a < p.na; ++a) {
        sr = cadd(sr, frame_sample(p.rc, q, p.xe, p.angles, p.starts, p.ns, p.nc, p.na, ch, a, 0, p.c, p.fs, p.fd, p.fn));
        sq = cadd(sq, frame_sample(p.cr, q, p.ye, p.angles, p.starts, p.ns, p.nc, p.na, ch, a, 1, p.c, p.fs, p.fd, p.fn));
      }
      sqrt_sum = cadd(sqrt_sum, cadd(csroot(sr), csroot(sq)));
      abs_sum += hypotf(sr.x, sr.y) + hypotf(sq.x, sq.y);
      bool ar, aq;
      receive_delay(q.x, q.z, double(p.xe[ch]), p.c, p.fn, &ar);
      receive_delay(q.y, q.z, double(p.ye[ch]), p.c, p.fn, &aq);
      active += float(ar) + float(aq);
    }
    float dm = cabs2(sqrt_sum) - abs_sum;
    float wc = (abs_sum > 0.f && active > 0.f) ? fmaxf(dm, 0.f) / active / abs_sum : 0.f;
    float inv = 1.0f / float(p.na);
    float2 mr = make_float2(rsum.x * inv, rsum.y * inv), mq = make_float2(qsum.x * inv, qsum.y * inv);
    float nr = cabs2(mr), nq = cabs2(mq);
    float var = fmaxf(er * inv - nr, 0.f) + fmaxf(eq * inv - nq, 0.f);
    float2 cx = cmul(mr, cconj(mq));
    float num = hypotf(cx.x, cx.y);
    float den = nr + nq + 0.5f * var - num;
    float wa = den > 0.f ? num / den : 0.f;
    float res = dm * wc * wa;
    dmas_out[v] = isfinite(res) ? res : 0.f;
  }
}

// Per-angle IQ (voxels, angles, frames) reductions of the single-frame API.
__global__ void angles_opw(const float2* iq, float2* out, size_t nv, size_t na, size_t nt) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nv * nt) return;
  size_t v = i / nt, t = i % nt;
  float2 acc = {};
  for (size_t a = 0; a < na; ++a) acc = cadd(acc, iq[(v * na + a) * nt + t]);
  out[i] = acc;
}

__global__ void angles_pd(const float2* iq, float* out, size_t nv, size_t na, size_t nt, size_t rs, size_t rn,
                          size_t cs, size_t cn, int fmas) {
  size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  float2 mean = {};
  float power = 0.f;
  for (size_t t = 0; t < nt; ++t) {
    float2 r = {}, q = {};
    for (size_t a = 0; a < rn; ++a) {
      float2 x = iq[(v * na + rs + a) * nt + t];
      r = cadd(r, fmas ? csroot(x) : x);
    }
    for (size_t a = 0; a < cn; ++a) {
      float2 x = iq[(v * na + cs + a) * nt + t];
      q = cadd(q, fmas ? csroot(x) : x);
    }
    if (fmas)
      power += cabs2(cmul(r, q));
    else
      mean = cadd(mean, cmul(r, cconj(q)));
  }
  out[v] = fmas ? power / float(nt) : hypotf(mean.x / float(nt), mean.y / float(nt));
}

}  // namespace generic
}  // namespace rcb
