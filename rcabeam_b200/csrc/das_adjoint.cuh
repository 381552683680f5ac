// Differentiable OPW delay-and-sum: forward with per-element delay offsets and
// a sound speed parameter, and its hand-written adjoint.
//
// Model (both apertures A = RC, CR; receive element e_c; offset d[A][c]):
//   tau   = (z cos th_a + u sin th_a) / c_s + sqrt(z^2 + (w - e_c)^2) / c_s + d[A][c]
//   s     = (tau - start_a) fs, valid iff 0 <= s <= ns - 1 and inside the f-number aperture
//   y     = ((1 - f) X[i0] + f X[i1]) exp(+j 2 pi fd tau),  i0 = floor(s), f = s - i0, i1 = min(i0 + 1, ns - 1)
//   IQ    = sum over A, c, a of y;  PD = mean_t |IQ|^2
// Adjoint, for the upstream gradient G = dL/dIQ (dL/dRe + j dL/dIm):
//   dX[i0] += (1 - f) conj(phase) G,  dX[i1] += f conj(phase) G          (scatter, atomics)
//   dL/dtau = Re sum_t conj(G) (fs (X[i1] - X[i0]) phase + j 2 pi fd y)
//   d offsets[A][c] += dL/dtau,  d c_s += dL/dtau * (-(tau - d[A][c]) / c_s)
// (reference model: src/rcabeam/sim.py:344-393 and opw.py:8-21; offsets and c_s
// are the parameters of the differentiation form).
//
// Both kernels work on a list of voxels and a chunk of at most kChunk frames,
// so the autograd layer recomputes IQ chunk by chunk in the backward pass
// instead of keeping the ensemble.  REAL = float reads complex64 channels and
// accumulates in float32 (phases from a float64-reduced cycle count, as the
// main path); REAL = double reads complex128 and is float64 throughout (the
// finite-difference checker).  Geometry is float64 in both.
#pragma once

#include "common.cuh"

namespace rcb {
namespace adj {

constexpr int kChunk = 8;  // frames per launch (registers per thread)

template <typename R>
struct Cx;
template <>
struct Cx<float> {
  using type = float2;
};
template <>
struct Cx<double> {
  using type = double2;
};

struct Geometry {
  const float* scan;
  const unsigned* voxels;  // list of voxel indices into scan, or null (identity)
  const float* xe;
  const float* ye;
  const float* angles;
  const float* starts;
  const double* offsets;  // [2][nc]
  double c, fs, fd, fn;
  int nvl, ns, nc, na, nt, f0, frames;
};

struct Tap64 {
  bool ok;
  int i0, i1;
  double tau, f;
};

__device__ __forceinline__ Tap64 tap(const Geometry& g, double u, double w, double z, int ap, int ch, int a) {
  Tap64 t;
  const double e = double(ap ? g.ye[ch] : g.xe[ch]);
  bool active = true;
  const double rx = receive_delay(w, z, e, g.c, g.fn, &active);
  const double th = double(g.angles[a]);
  t.tau = __dadd_rn(__dadd_rn(transmit_delay(u, z, cos(th), sin(th), g.c), rx), g.offsets[ap * g.nc + ch]);
  const double s = __dmul_rn(__dadd_rn(t.tau, -double(g.starts[a])), g.fs);
  t.ok = active && s >= 0.0 && s <= double(g.ns - 1);
  const double fl = floor(s);
  t.i0 = t.ok ? int(fl) : 0;
  t.i1 = min(t.i0 + 1, g.ns - 1);
  t.f = s - fl;
  return t;
}

template <typename R>
__device__ __forceinline__ typename Cx<R>::type phase_of(double fd, double tau) {
  double cyc = fd * tau;
  cyc -= rint(cyc);
  if constexpr (sizeof(R) == 4) {
    float sn, cs;
    sincospif(2.0f * float(cyc), &sn, &cs);
    return make_float2(cs, sn);
  } else {
    double sn, cs;
    sincospi(2.0 * cyc, &sn, &cs);
    return make_double2(cs, sn);
  }
}

__device__ __forceinline__ void voxel_pos(const Geometry& g, int l, double& x, double& z, double& y) {
  const size_t v = g.voxels ? size_t(g.voxels[l]) : size_t(l);
  x = double(g.scan[3 * v]);
  z = double(g.scan[3 * v + 1]);
  y = double(g.scan[3 * v + 2]);
}

// One thread per listed voxel: IQ of frames [f0, f0 + frames) and/or its power sum.
template <typename R>
__global__ void __launch_bounds__(128) forward(Geometry g, const typename Cx<R>::type* __restrict__ rc,
                                               const typename Cx<R>::type* __restrict__ cr,
                                               typename Cx<R>::type* __restrict__ iq, double* __restrict__ power) {
  using C = typename Cx<R>::type;
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= g.nvl) return;
  double x, z, y;
  voxel_pos(g, l, x, z, y);
  R re[kChunk], im[kChunk];
#pragma unroll
  for (int t = 0; t < kChunk; ++t) re[t] = im[t] = R(0);
  for (int ap = 0; ap < 2; ++ap) {
    const C* X = ap ? cr : rc;
    const double u = ap ? x : y, w = ap ? y : x;
    for (int ch = 0; ch < g.nc; ++ch) {
      for (int a = 0; a < g.na; ++a) {
        const Tap64 t = tap(g, u, w, z, ap, ch, a);
        if (!t.ok) continue;
        const C ph = phase_of<R>(g.fd, t.tau);
        const R f = R(t.f), f0w = R(1) - f;
        const size_t b0 = ((size_t(t.i0) * g.nc + ch) * g.na + a) * g.nt + g.f0;
        const size_t b1 = ((size_t(t.i1) * g.nc + ch) * g.na + a) * g.nt + g.f0;
#pragma unroll
        for (int k = 0; k < kChunk; ++k) {
          if (k < g.frames) {
            const C x0 = X[b0 + k], x1 = X[b1 + k];
            const R vr = f0w * x0.x + f * x1.x, vi = f0w * x0.y + f * x1.y;
            re[k] += vr * ph.x - vi * ph.y;
            im[k] += vr * ph.y + vi * ph.x;
          }
        }
      }
    }
  }
  double p = 0.0;
#pragma unroll
  for (int k = 0; k < kChunk; ++k) {
    if (k < g.frames) {
      if (iq) iq[size_t(l) * g.frames + k] = C{re[k], im[k]};
      p += double(re[k]) * double(re[k]) + double(im[k]) * double(im[k]);
    }
  }
  if (power) power[l] += p / double(g.nt);
}

__device__ __forceinline__ void atomic_add_c(float2* p, float2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}
__device__ __forceinline__ void atomic_add_c(double2* p, double2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}

// One thread per (listed voxel, aperture, channel): scatter of G into the
// channel gradients and the delay / sound-speed gradient sums.
template <typename R>
__global__ void __launch_bounds__(128) adjoint(Geometry g, const typename Cx<R>::type* __restrict__ rc,
                                               const typename Cx<R>::type* __restrict__ cr,
                                               const typename Cx<R>::type* __restrict__ grad_iq,
                                               typename Cx<R>::type* grad_rc, typename Cx<R>::type* grad_cr,
                                               double* grad_offsets, double* grad_c) {
  using C = typename Cx<R>::type;
  const size_t id = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t total = size_t(g.nvl) * 2 * g.nc;
  double d_tau_sum = 0.0, d_c = 0.0;
  int ap = 0, ch = 0;
  if (id < total) {
    const int l = int(id / (2 * g.nc));
    ap = int((id / g.nc) % 2);
    ch = int(id % g.nc);
    double x, z, y;
    voxel_pos(g, l, x, z, y);
    const C* X = ap ? cr : rc;
    C* GX = ap ? grad_cr : grad_rc;
    const double u = ap ? x : y, w = ap ? y : x;
    C G[kChunk];
#pragma unroll
    for (int k = 0; k < kChunk; ++k) G[k] = k < g.frames ? grad_iq[size_t(l) * g.frames + k] : C{R(0), R(0)};
    const double two_pi_fd = 2.0 * 3.141592653589793 * g.fd;
    for (int a = 0; a < g.na; ++a) {
      const Tap64 t = tap(g, u, w, z, ap, ch, a);
      if (!t.ok) continue;
      const C ph = phase_of<R>(g.fd, t.tau);
      const R f = R(t.f), f0w = R(1) - f;
      const size_t b0 = ((size_t(t.i0) * g.nc + ch) * g.na + a) * g.nt + g.f0;
      const size_t b1 = ((size_t(t.i1) * g.nc + ch) * g.na + a) * g.nt + g.f0;
      double dtau = 0.0;
#pragma unroll
      for (int k = 0; k < kChunk; ++k) {
        if (k < g.frames) {
          const C x0 = X[b0 + k], x1 = X[b1 + k];
          // conj(phase) G, weighted onto the two taps.
          const R cr_ = ph.x * G[k].x + ph.y * G[k].y, ci = ph.x * G[k].y - ph.y * G[k].x;
          atomic_add_c(GX + b0 + k, C{f0w * cr_, f0w * ci});
          atomic_add_c(GX + b1 + k, C{f * cr_, f * ci});
          // y and its tau derivative.
          const double vr = double(f0w) * x0.x + double(f) * x1.x, vi = double(f0w) * x0.y + double(f) * x1.y;
          const double yr = vr * ph.x - vi * ph.y, yi = vr * ph.y + vi * ph.x;
          const double sr = g.fs * (double(x1.x) - x0.x), si = g.fs * (double(x1.y) - x0.y);
          const double dr = sr * ph.x - si * ph.y - two_pi_fd * yi;
          const double di = sr * ph.y + si * ph.x + two_pi_fd * yr;
          dtau += double(G[k].x) * dr + double(G[k].y) * di;  // Re(conj(G) dy)
        }
      }
      d_tau_sum += dtau;
      d_c += dtau * (-(t.tau - g.offsets[ap * g.nc + ch]) / g.c);
    }
    if (d_tau_sum != 0.0) atomicAdd(grad_offsets + ap * g.nc + ch, d_tau_sum);
  }
  for (int off = 16; off > 0; off >>= 1) d_c += __shfl_xor_sync(0xffffffffu, d_c, off);
  if ((threadIdx.x & 31) == 0 && d_c != 0.0) atomicAdd(grad_c, d_c);
}

}  // namespace adj
}  // namespace rcb
