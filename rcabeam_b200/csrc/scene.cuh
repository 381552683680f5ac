// Forward model of RCA channel IQ for seeded point-scatterer scenes.
//
// Each scatterer k moves along a line: position(t) = o_k + d_k s_k(t), with
// s_k(t) = s0_k + speed_k t, wrapped into [0, period_k) when period_k > 0 (a
// scatterer flowing through a tube re-enters at its start).  Frame f is
// acquired at t = f / prf.  The channel sample of (sample i, element e, angle a,
// frame f) is the sum over scatterers of
//
//     amp_k exp(-((t_i - tau)/sigma)^2) exp(-j 2 pi fd tau),   t_i = start_a + i / fs,
//     tau = (z cos(theta_a) + u sin(theta_a)) / c + sqrt(z^2 + (v - e)^2) / c
//
// with v = x, u = y for RC and v = y, u = x for CR: the Gaussian-pulse model of
// the reference's simulate_point (src/rcabeam/sim.py:131-189, sigma_t branch),
// evaluated only where |t_i - tau| <= half_width.  Delays are float64.
//
// One CTA per (element, angle, frame chunk) accumulates its (samples x chunk)
// slab in shared memory; threads take (scatterer, frame) pairs.  Every output
// element is written exactly once, so the output needs no clearing.
#pragma once

#include "common.cuh"

namespace rcb {
namespace scene {

constexpr int kThreads = 256;
constexpr int kFields = 11;  // ox, oz, oy, dx, dz, dy, s0, speed, period, amp_re, amp_im

struct Args {
  const float* scatterers;  // n x kFields
  size_t n;
  const float* elements;    // receive elements of this aperture
  const float* angles;
  const float* starts;
  float2* out;              // (ns, nc, na, nt) complex64
  int ns, nc, na, nt, chunk;
  int config;               // 0 = RC, 1 = CR
  double prf, c, fs, fd, sigma, half_width;
};

__global__ void __launch_bounds__(kThreads) simulate(Args p) {
  extern __shared__ float2 slab[];  // [ns][chunk]
  const int ch = blockIdx.x / p.na, a = blockIdx.x % p.na;
  const int f0 = blockIdx.y * p.chunk;
  const int nf = min(p.chunk, p.nt - f0);
  for (int i = threadIdx.x; i < p.ns * p.chunk; i += blockDim.x) slab[i] = make_float2(0.f, 0.f);
  __syncthreads();
  const double e = double(p.elements[ch]);
  const double th = double(p.angles[a]);
  const double cs = cos(th), sn = sin(th);
  const double start = double(p.starts[a]);
  const size_t pairs = p.n * size_t(nf);
  for (size_t q = threadIdx.x; q < pairs; q += blockDim.x) {
    const size_t k = q / size_t(nf);
    const int f = int(q - k * size_t(nf));
    const float* s = p.scatterers + k * kFields;
    const double t = double(f0 + f) / p.prf;
    double along = double(s[6]) + double(s[7]) * t;
    const double period = double(s[8]);
    if (period > 0.0) along -= period * floor(along / period);
    const double x = double(s[0]) + double(s[3]) * along;
    const double z = double(s[1]) + double(s[4]) * along;
    const double y = double(s[2]) + double(s[5]) * along;
    const double v = p.config ? y : x, u = p.config ? x : y;
    const double d = v - e;
    const double tau = (z * cs + u * sn) / p.c + sqrt(z * z + d * d) / p.c;
    const double center = (tau - start) * p.fs;
    const double reach = p.half_width * p.fs;
    const int lo = max(0, int(ceil(center - reach)));
    const int hi = min(p.ns - 1, int(floor(center + reach)));
    if (lo > hi) continue;
    double cyc = p.fd * tau;
    cyc -= rint(cyc);
    float sine, cosine;
    sincospif(-2.0f * float(cyc), &sine, &cosine);
    const float2 amp = make_float2(s[9], s[10]);
    const float2 rot = make_float2(amp.x * cosine - amp.y * sine, amp.x * sine + amp.y * cosine);
    for (int i = lo; i <= hi; ++i) {
      const float r = float((start + double(i) / p.fs - tau) / p.sigma);
      const float env = expf(-r * r);
      float2* dst = slab + size_t(i) * p.chunk + f;
      atomicAdd(&dst->x, rot.x * env);
      atomicAdd(&dst->y, rot.y * env);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < p.ns * nf; i += blockDim.x) {
    const int row = i / nf, f = i - row * nf;
    p.out[((size_t(row) * p.nc + ch) * p.na + a) * p.nt + f0 + f] = slab[size_t(row) * p.chunk + f];
  }
}

}  // namespace scene
}  // namespace rcb
