/* Float64 RCA delay-and-sum oracle in C -- TEST INFRASTRUCTURE ONLY.
 *
 * The same arithmetic as oracle/das.py:aperture_das, which restates the
 * reference's NumPy DAS _delay_numpy (src/rcabeam/sim.py:344-393):
 *   tau_rx = sqrt(z^2 + (v - e)^2) / c (+ offset), v = x (RC) or y (CR)   sim.py:369-371
 *   tau_tx = (z cos(theta) + u sin(theta)) / c, u = y (RC) or x (CR)     sim.py:369, 377
 *   sample = (tau - start[a]) fs, valid iff 0 <= sample <= ns - 1          sim.py:379-380
 *   lower = floor(clip(sample)), upper = min(lower + 1, ns - 1),
 *   w = clip(sample) - lower, value = (1 - w) x[lower] + w x[upper]       sim.py:381-384
 *   value * exp(+j 2 pi fd tau), masked by |v - e| <= z / (2 fnumber)      sim.py:373, 385
 * summed over channels and angles into out (sim.py:386; opw.py:8-21), all in
 * float64.  It exists because the NumPy restatement needs tens of seconds for
 * a 65,536-voxel grid; this one runs threaded over voxels (OpenMP) and is
 * checked against the NumPy restatement in the CPU tests.
 *
 * iq: complex64 (ns, nc, na, nt) as interleaved floats; scan: (nv, 3) float64
 * (x, z, y); out: (nv, nt) complex128 as interleaved doubles, ACCUMULATED. */
#include <math.h>
#include <stddef.h>

void oracle_das_accumulate(const float* iq, const double* scan, size_t nv, const double* elements,
                           const double* angles, const double* starts, const double* offsets, size_t ns, size_t nc,
                           size_t na, size_t nt, double c, double fs, double fd, double fnumber, int config,
                           double* out) {
  const int full = !(fnumber > 0.0);
  const double two_pi = 2.0 * M_PI;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long vi = 0; vi < (long long)nv; ++vi) {
    const double x = scan[3 * vi], z = scan[3 * vi + 1], y = scan[3 * vi + 2];
    const double v_rx = config ? y : x, u_tx = config ? x : y;
    double* dst = out + 2 * (size_t)vi * nt;
    for (size_t ch = 0; ch < nc; ++ch) {
      const double distance = v_rx - elements[ch];
      const double receive = sqrt(z * z + distance * distance) / c + (offsets ? offsets[ch] : 0.0);
      const int active = full || fabs(distance) <= z / (2.0 * fnumber);
      if (!active) continue;
      for (size_t a = 0; a < na; ++a) {
        const double transmit = (z * cos(angles[a]) + u_tx * sin(angles[a])) / c;
        const double tau = transmit + receive;
        const double sample = (tau - starts[a]) * fs;
        if (!(sample >= 0.0) || !(sample <= (double)(ns - 1))) continue;
        const double lower_f = floor(sample);
        const size_t lower = (size_t)lower_f;
        const size_t upper = lower + 1 < ns ? lower + 1 : ns - 1;
        const double w = sample - lower_f;
        const double arg = two_pi * fd * tau;
        const double pr = cos(arg), pi = sin(arg);
        const float* xa = iq + 2 * ((lower * nc + ch) * na + a) * nt;
        const float* xb = iq + 2 * ((upper * nc + ch) * na + a) * nt;
        for (size_t t = 0; t < nt; ++t) {
          const double vr = (1.0 - w) * (double)xa[2 * t] + w * (double)xb[2 * t];
          const double vim = (1.0 - w) * (double)xa[2 * t + 1] + w * (double)xb[2 * t + 1];
          dst[2 * t] += vr * pr - vim * pi;
          dst[2 * t + 1] += vr * pi + vim * pr;
        }
      }
    }
  }
}
