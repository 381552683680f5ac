// Global temporal SVD clutter filter kernels (reference src/rcabeam/gpu_clutter.py).
//
//   * scale:  max |component| of the Casorati matrix (gpu_clutter.py:141);
//   * gram:   G = (X / s)^H (X / s) / rows over the upper triangle of 64 x 64
//             frame tiles, split over row slices; CUDA-core float64 (the
//             reference default) or float32 accumulation (its complex64 mode);
//   * finish: Hermitian symmetrization into a column-major complex128 matrix;
//   * project: per row, coordinates y = x V on k temporal vectors, then either
//             the retained power sum |y|^2 / T or the residual x - y V^H
//             (written out and/or reduced to power), float64 throughout
//             (gpu_clutter.py:196-273).
// The tensor-core Gram forms live in gram_tc.cuh.
#pragma once

#include "common.cuh"

namespace rcb {
namespace clutter {

constexpr int kGramTile = 64;     // frame columns per Gram tile
constexpr int kGramRows = 16;     // rows staged per iteration
constexpr int kGramThreads = 256; // 16 x 16 threads, 4 x 4 complex outputs each

template <typename T>
struct Cx;
template <>
struct Cx<float> {
  using type = float2;
};
template <>
struct Cx<double> {
  using type = double2;
};

template <typename IN>
__device__ __forceinline__ double2 load_c(const IN* p, size_t i) {
  if constexpr (sizeof(IN) == 8) {
    float2 v = reinterpret_cast<const float2*>(p)[i];
    return make_double2(v.x, v.y);
  } else {
    return reinterpret_cast<const double2*>(p)[i];
  }
}

// Max over |re| and |im| (non-negative doubles order like their bit patterns).
// A NaN component makes the result a quiet NaN (whose bits order above +inf
// in the unsigned maximum), so a non-finite input always gives a non-finite
// scale: the caller's finite-input check reads the scale instead of the input.
constexpr unsigned long long kNanBits = 0x7ff8000000000000ull;

template <typename IN>
__global__ void max_abs_kernel(const IN* x, size_t n, unsigned long long* out) {
  double m = 0.0;
  bool nan = false;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    double2 v = load_c(x, i);
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    nan |= isnan(v.x) || isnan(v.y);
  }
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  const unsigned long long bits = __any_sync(0xffffffffu, nan) ? kNanBits : __double_as_longlong(m);
  if ((threadIdx.x & 31) == 0) atomicMax(out, bits);
}

// Complex64 max |component| at HBM speed: float4 loads (two samples), four in
// flight per thread; the float maximum is exact, so the result equals
// max_abs_kernel's.  x must be 16-byte aligned; an odd last sample is read alone.
__global__ void __launch_bounds__(256) max_abs_c64(const float2* __restrict__ x, size_t n,
                                                   unsigned long long* out) {
  const float4* x4 = reinterpret_cast<const float4*>(x);
  const size_t n4 = n / 2, stride = size_t(gridDim.x) * blockDim.x;
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  float m = 0.f;
  bool nan = false;
  auto fold = [&m, &nan](float4 v) {
    m = fmaxf(fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y))), fmaxf(fabsf(v.z), fabsf(v.w)));
    nan |= isnan(v.x) || isnan(v.y) || isnan(v.z) || isnan(v.w);
  };
  for (; i + 3 * stride < n4; i += 4 * stride) {
    const float4 a = __ldg(x4 + i), b = __ldg(x4 + i + stride), c = __ldg(x4 + i + 2 * stride),
                 d = __ldg(x4 + i + 3 * stride);
    fold(a);
    fold(b);
    fold(c);
    fold(d);
  }
  for (; i < n4; i += stride) fold(__ldg(x4 + i));
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const float2 t = x[n - 1];
    m = fmaxf(m, fmaxf(fabsf(t.x), fabsf(t.y)));
    nan |= isnan(t.x) || isnan(t.y);
  }
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  const unsigned long long bits =
      __any_sync(0xffffffffu, nan) ? kNanBits : static_cast<unsigned long long>(__double_as_longlong(double(m)));
  if ((threadIdx.x & 31) == 0) atomicMax(out, bits);
}

// Partial Gram of one upper-triangle tile (bi <= bj) over a slice of rows.
// Each thread owns a 4 x 4 block of complex outputs; rows are staged through
// shared memory already scaled and converted to the accumulation type.
template <typename ACC, typename IN>
__global__ void __launch_bounds__(kGramThreads)
    gram_simt(const IN* __restrict__ x, size_t rows, int nt, const double* __restrict__ scale,
              int tiles_per_row_block, double* __restrict__ gram) {
  using C = typename Cx<ACC>::type;
  __shared__ C si[kGramRows][kGramTile];
  __shared__ C sj[kGramRows][kGramTile];
  // Map blockIdx.x to the (bi, bj) upper-triangle tile.
  int t = blockIdx.x, bi = 0;
  int nb = tiles_per_row_block;
  while (t >= nb - bi) {
    t -= nb - bi;
    ++bi;
  }
  const int bj = bi + t;
  const int ti = threadIdx.x / 16, tj = threadIdx.x % 16;
  const size_t slices = gridDim.y;
  const size_t per = (rows + slices - 1) / slices;
  const size_t r0 = blockIdx.y * per, r1 = min(rows, r0 + per);
  ACC acc_r[4][4] = {}, acc_i[4][4] = {};
  const ACC s = ACC(*scale > 0.0 ? 1.0 / *scale : 1.0);
  for (size_t base = r0; base < r1; base += kGramRows) {
    for (int e = threadIdx.x; e < kGramRows * kGramTile; e += kGramThreads) {
      int rr = e / kGramTile, cc = e % kGramTile;
      size_t r = base + rr;
      int ci = bi * kGramTile + cc, cj = bj * kGramTile + cc;
      double2 vi = (r < r1 && ci < nt) ? load_c(x, r * nt + ci) : make_double2(0.0, 0.0);
      double2 vj = (r < r1 && cj < nt) ? load_c(x, r * nt + cj) : make_double2(0.0, 0.0);
      si[rr][cc] = C{ACC(vi.x) * s, ACC(vi.y) * s};
      sj[rr][cc] = C{ACC(vj.x) * s, ACC(vj.y) * s};
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < kGramRows; ++rr) {
      C a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = si[rr][ti + 16 * u];
        b[u] = sj[rr][tj + 16 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          // conj(a) * b
          acc_r[u][v] = fma(a[u].x, b[v].x, fma(a[u].y, b[v].y, acc_r[u][v]));
          acc_i[u][v] = fma(a[u].x, b[v].y, fma(-a[u].y, b[v].x, acc_i[u][v]));
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      int i = bi * kGramTile + ti + 16 * u, j = bj * kGramTile + tj + 16 * v;
      if (i < nt && j < nt) {
        atomicAdd(gram + 2 * (size_t(i) * nt + j), double(acc_r[u][v]));
        atomicAdd(gram + 2 * (size_t(i) * nt + j) + 1, double(acc_i[u][v]));
      }
    }
  }
}

// Row-major upper-triangle partial sums -> column-major Hermitian complex128
// matrix divided by rows: out = (G + G^H) / (2 rows) (gpu_clutter.py:161).
__global__ void gram_finish(const double* upper, double* out, int nt, double inv_rows) {
  int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nt) return;
  int bi = i / kGramTile, bj = j / kGramTile;
  // Entries of tiles below the diagonal were never accumulated: use conj(G[j][i]).
  double2 gij = make_double2(0.0, 0.0), gji = make_double2(0.0, 0.0);
  bool have_ij = bi <= bj, have_ji = bj <= bi;
  if (have_ij) gij = make_double2(upper[2 * (size_t(i) * nt + j)], upper[2 * (size_t(i) * nt + j) + 1]);
  if (have_ji) gji = make_double2(upper[2 * (size_t(j) * nt + i)], upper[2 * (size_t(j) * nt + i) + 1]);
  if (!have_ij) gij = make_double2(gji.x, -gji.y);
  if (!have_ji) gji = make_double2(gij.x, -gij.y);
  double re = 0.5 * (gij.x + gji.x) * inv_rows;
  double im = 0.5 * (gij.y - gji.y) * inv_rows;
  // Column-major: element (i, j) at i + j * nt.
  out[2 * (size_t(j) * nt + i)] = re;
  out[2 * (size_t(j) * nt + i) + 1] = im;
}

constexpr int kProjChunk = 8;  // temporal vectors per register chunk

// One warp per row.  vec: T x k complex128, column-major (vec[t + c * T]).
// mode bit 0: subtract (residual x - (x V) V^H) else retained coordinates only;
// bit 1: write filtered rows (same dtype as the input); power always written when non-null.
template <typename IN, int MAXF>
__global__ void __launch_bounds__(256)
    project_rows(const IN* __restrict__ x, IN* __restrict__ out, double* __restrict__ power, size_t rows, int nt,
                 const double2* __restrict__ vec, int k, int mode, double inv_nt) {
  const int lane = threadIdx.x & 31;
  const size_t row = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
  if (row >= rows) return;
  double2 xv[MAXF], proj[MAXF];
#pragma unroll
  for (int f = 0; f < MAXF; ++f) {
    int t = lane + 32 * f;
    xv[f] = t < nt ? load_c(x, row * nt + t) : make_double2(0.0, 0.0);
    proj[f] = make_double2(0.0, 0.0);
  }
  double retained = 0.0;
  for (int c0 = 0; c0 < k; c0 += kProjChunk) {
    double2 y[kProjChunk];
#pragma unroll
    for (int c = 0; c < kProjChunk; ++c) {
      double yr = 0.0, yi = 0.0;
      if (c0 + c < k) {
#pragma unroll
        for (int f = 0; f < MAXF; ++f) {
          int t = lane + 32 * f;
          if (t < nt) {
            double2 v = vec[t + size_t(c0 + c) * nt];
            yr = fma(xv[f].x, v.x, fma(-xv[f].y, v.y, yr));
            yi = fma(xv[f].x, v.y, fma(xv[f].y, v.x, yi));
          }
        }
      }
      if (c0 + c < k) {  // k is uniform over the warp: slots past k reduce nothing
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          yr += __shfl_xor_sync(0xffffffffu, yr, off);
          yi += __shfl_xor_sync(0xffffffffu, yi, off);
        }
      }
      y[c] = make_double2(yr, yi);
      retained += yr * yr + yi * yi;
    }
    if (mode & 3) {
#pragma unroll
      for (int f = 0; f < MAXF; ++f) {
        int t = lane + 32 * f;
        if (t < nt) {
#pragma unroll
          for (int c = 0; c < kProjChunk; ++c) {
            if (c0 + c < k) {
              // y * conj(v)
              double2 v = vec[t + size_t(c0 + c) * nt];
              proj[f].x = fma(y[c].x, v.x, fma(y[c].y, v.y, proj[f].x));
              proj[f].y = fma(y[c].y, v.x, fma(-y[c].x, v.y, proj[f].y));
            }
          }
        }
      }
    }
  }
  const bool subtract = mode & 1;
  double pw = 0.0;
#pragma unroll
  for (int f = 0; f < MAXF; ++f) {
    int t = lane + 32 * f;
    if (t < nt) {
      double2 r = subtract ? make_double2(xv[f].x - proj[f].x, xv[f].y - proj[f].y) : proj[f];
      pw += r.x * r.x + r.y * r.y;
      if (mode & 2) {
        if constexpr (sizeof(IN) == 8)
          reinterpret_cast<float2*>(out)[row * nt + t] = make_float2(float(r.x), float(r.y));
        else
          reinterpret_cast<double2*>(out)[row * nt + t] = r;
      }
    }
  }
  if (power) {
    if (subtract) {
      for (int off = 16; off > 0; off >>= 1) pw += __shfl_xor_sync(0xffffffffu, pw, off);
      if (lane == 0) power[row] = pw * inv_nt;
    } else if (lane == 0) {
      power[row] = retained * inv_nt;
    }
  }
}

constexpr int kProjSmall = 4;  // vectors of the single-chunk form

// Single-chunk form of project_rows (k <= kProjSmall, the usual case): the
// projection of each frame is formed on the fly in the final pass from the k
// reduced coordinates, so no per-frame projection array is held, and the row
// stays in registers in its input precision (widened exactly where used).
// Same operations in the same order as project_rows, so the same results, with
// about half the registers (more resident warps for this latency-bound pass).
template <typename IN, int MAXF>
__global__ void __launch_bounds__(128)
    project_rows_one(const IN* __restrict__ x, IN* __restrict__ out, double* __restrict__ power, size_t rows,
                     int nt, const double2* __restrict__ vec, int k, int mode, double inv_nt) {
  const int lane = threadIdx.x & 31;
  const size_t row = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
  if (row >= rows) return;
  IN xv[MAXF];
#pragma unroll
  for (int f = 0; f < MAXF; ++f) {
    const int t = lane + 32 * f;
    xv[f] = t < nt ? x[row * nt + t] : IN{};
  }
  double2 y[kProjSmall];
  double retained = 0.0;
#pragma unroll
  for (int c = 0; c < kProjSmall; ++c) {
    double yr = 0.0, yi = 0.0;
    if (c < k) {  // k is uniform over the warp
#pragma unroll
      for (int f = 0; f < MAXF; ++f) {
        const int t = lane + 32 * f;
        if (t < nt) {
          const double2 v = vec[t + size_t(c) * nt];
          const double xr = double(xv[f].x), xi = double(xv[f].y);
          yr = fma(xr, v.x, fma(-xi, v.y, yr));
          yi = fma(xr, v.y, fma(xi, v.x, yi));
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        yr += __shfl_xor_sync(0xffffffffu, yr, off);
        yi += __shfl_xor_sync(0xffffffffu, yi, off);
      }
    }
    y[c] = make_double2(yr, yi);
    retained += yr * yr + yi * yi;
  }
  const bool subtract = mode & 1;
  double pw = 0.0;
  if (mode & 3) {
#pragma unroll
    for (int f = 0; f < MAXF; ++f) {
      const int t = lane + 32 * f;
      if (t < nt) {
        double2 proj = make_double2(0.0, 0.0);
#pragma unroll
        for (int c = 0; c < kProjSmall; ++c) {
          if (c < k) {  // y * conj(v)
            const double2 v = vec[t + size_t(c) * nt];
            proj.x = fma(y[c].x, v.x, fma(y[c].y, v.y, proj.x));
            proj.y = fma(y[c].y, v.x, fma(-y[c].x, v.y, proj.y));
          }
        }
        const double2 r =
            subtract ? make_double2(double(xv[f].x) - proj.x, double(xv[f].y) - proj.y) : proj;
        pw += r.x * r.x + r.y * r.y;
        if (mode & 2) {
          if constexpr (sizeof(IN) == 8)
            reinterpret_cast<float2*>(out)[row * nt + t] = make_float2(float(r.x), float(r.y));
          else
            reinterpret_cast<double2*>(out)[row * nt + t] = r;
        }
      }
    }
  }
  if (power) {
    if (subtract) {
      for (int off = 16; off > 0; off >>= 1) pw += __shfl_xor_sync(0xffffffffu, pw, off);
      if (lane == 0) power[row] = pw * inv_nt;
    } else if (lane == 0) {
      power[row] = retained * inv_nt;
    }
  }
}

// Persistent form of the small projection (k <= kProjSmall): one warp per row,
// lane l holding frames l, l + 32, ... widened to float64 once, in registers.
// Each warp keeps its next kAsyncDepth - 1 rows in flight with cp.async
// (8-byte copies for complex64, 16-byte for complex128) into a per-warp
// shared-memory ring, so the bytes in flight per SM do not cost registers; a
// lane reads back only the frames it copied itself, so no warp barrier is
// needed.  The k vectors are staged in shared memory once per CTA.  Same sums
// in the same order as project_rows_one.  flags (optional): bit 0 is set when
// an input component is not finite, bit 1 when a row's power is not finite.
constexpr int kAsyncThreads = 256;
constexpr int kAsyncWarps = kAsyncThreads / 32;
constexpr int kAsyncDepth = 3;

__host__ __device__ inline size_t async_smem_bytes(size_t k, size_t nt, size_t elem) {
  return (k * nt * 16 + 15) / 16 * 16 + size_t(kAsyncWarps) * kAsyncDepth * nt * elem;
}

template <typename IN>
__device__ __forceinline__ void async_copy(IN* dst, const IN* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  if constexpr (sizeof(IN) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

template <typename IN, int MAXF>
__global__ void __launch_bounds__(kAsyncThreads, 2)
    project_rows_async(const IN* __restrict__ x, IN* __restrict__ out, double* __restrict__ power, size_t rows,
                       int nt, const double2* __restrict__ vec, int k, int mode, double inv_nt,
                       unsigned* __restrict__ flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* vs = reinterpret_cast<double2*>(smem);  // [k][nt]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  IN* ring = reinterpret_cast<IN*>(smem + (size_t(k) * nt * 16 + 15) / 16 * 16) + size_t(warp) * kAsyncDepth * nt;
  for (int i = threadIdx.x; i < k * nt; i += blockDim.x) vs[i] = vec[i];
  __syncthreads();
  const size_t stride = size_t(gridDim.x) * kAsyncWarps;
  size_t row = size_t(blockIdx.x) * kAsyncWarps + warp;
  auto issue = [&](size_t r, int slot) {
    if (r < rows) {
#pragma unroll
      for (int f = 0; f < MAXF; ++f) {
        const int t = lane + 32 * f;
        if (t < nt) async_copy(ring + slot * nt + t, x + r * nt + t);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
#pragma unroll
  for (int d = 0; d < kAsyncDepth - 1; ++d) issue(row + d * stride, d);
  const bool subtract = mode & 1;
  bool bad_in = false, bad_out = false;
  for (int i = 0; row < rows; ++i, row += stride) {
    issue(row + (kAsyncDepth - 1) * stride, (i + kAsyncDepth - 1) % kAsyncDepth);
    asm volatile("cp.async.wait_group %0;" ::"n"(kAsyncDepth - 1) : "memory");
    const IN* cur = ring + (i % kAsyncDepth) * nt;
    double2 xv[MAXF];
#pragma unroll
    for (int f = 0; f < MAXF; ++f) {
      const int t = lane + 32 * f;
      if (t < nt) {
        const IN a = cur[t];
        xv[f] = make_double2(double(a.x), double(a.y));
        bad_in |= !isfinite(xv[f].x) || !isfinite(xv[f].y);
      } else {
        xv[f] = make_double2(0.0, 0.0);
      }
    }
    double2 y[kProjSmall];
    double retained = 0.0;
#pragma unroll
    for (int c = 0; c < kProjSmall; ++c) {
      double yr = 0.0, yi = 0.0;
      if (c < k) {
#pragma unroll
        for (int f = 0; f < MAXF; ++f) {
          const int t = lane + 32 * f;
          if (t < nt) {
            const double2 v = vs[c * nt + t];
            yr = fma(xv[f].x, v.x, fma(-xv[f].y, v.y, yr));
            yi = fma(xv[f].x, v.y, fma(xv[f].y, v.x, yi));
          }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          yr += __shfl_xor_sync(0xffffffffu, yr, off);
          yi += __shfl_xor_sync(0xffffffffu, yi, off);
        }
      }
      y[c] = make_double2(yr, yi);
      retained += yr * yr + yi * yi;
    }
    double pw = 0.0;
    if (mode & 3) {
#pragma unroll
      for (int f = 0; f < MAXF; ++f) {
        const int t = lane + 32 * f;
        if (t < nt) {
          double2 proj = make_double2(0.0, 0.0);
#pragma unroll
          for (int c = 0; c < kProjSmall; ++c) {
            if (c < k) {  // y * conj(v)
              const double2 v = vs[c * nt + t];
              proj.x = fma(y[c].x, v.x, fma(y[c].y, v.y, proj.x));
              proj.y = fma(y[c].y, v.x, fma(-y[c].x, v.y, proj.y));
            }
          }
          const double2 r = subtract ? make_double2(xv[f].x - proj.x, xv[f].y - proj.y) : proj;
          pw += r.x * r.x + r.y * r.y;
          if (mode & 2) {
            if constexpr (sizeof(IN) == 8)
              reinterpret_cast<float2*>(out)[row * nt + t] = make_float2(float(r.x), float(r.y));
            else
              reinterpret_cast<double2*>(out)[row * nt + t] = r;
          }
        }
      }
    }
    if (power) {
      if (subtract) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) pw += __shfl_xor_sync(0xffffffffu, pw, off);
      } else {
        pw = retained;
      }
      if (lane == 0) {
        power[row] = pw * inv_nt;
        bad_out |= !isfinite(pw);
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  if (flags) {
    const unsigned bits = (__any_sync(0xffffffffu, bad_in) ? 1u : 0u) | (__any_sync(0xffffffffu, bad_out) ? 2u : 0u);
    if (bits && lane == 0) atomicOr(flags, bits);
  }
}

// Register form of project_rows_async for complex64 rows, K <= 3 vectors and
// nt <= 32 F: lane l holds the vectors' values at its frames l, l + 32, ...
// in registers for the whole launch, so a row costs its samples' read and
// float64 arithmetic only (the shared-memory form reads 2 K F double2 per
// lane and row back, about twice the shared-memory cycles its float64 work
// takes).  The coordinates' warp sums run as one reduce-scatter
// (warp_sum_coordinates), so their float64 sum order differs from
// project_rows_async's butterflies (last-bit differences).
// H = 2 extends it to 256 < nt <= 512: a row per pair of warps, warp h of the
// pair holding frames 32 F h + l + 32 f; the pair adds its two partial
// coordinates (and partial powers) through shared memory behind a 64-thread
// named barrier, half 0 first in both warps.
constexpr int kRegThreads = 128;
constexpr int kRegWarps = kRegThreads / 32;

// Warp sums of the 2K partial coordinate components (re, im of each vector),
// returned to every lane: a reduce-scatter over the padded power of two P of
// components (at each of the first log2 P xor levels a lane keeps the half its
// lane bit selects and receives the partner's partial of that half; P - 1
// shuffles), butterflies over the remaining levels for the one component a
// lane then holds, and a gather from the lanes 4i that hold component i.  For
// K = 3 that is 15 float64 shuffles per row instead of 30 for six butterfly
// sums.
template <int K>
__device__ __forceinline__ void warp_sum_coordinates(const double (&part)[2 * K], int lane, double2 (&y)[K]) {
  constexpr int V = 2 * K;
  constexpr int P = V <= 2 ? 2 : V <= 4 ? 4 : 8;
  constexpr int L = P == 2 ? 1 : P == 4 ? 2 : 3;  // reduce-scatter levels
  double w[P];
#pragma unroll
  for (int i = 0; i < P; ++i) w[i] = i < V ? part[i] : 0.0;
#pragma unroll
  for (int l = 0; l < L; ++l) {
    const int off = 16 >> l, half = (P >> l) / 2;
    const bool upper = lane & off;
#pragma unroll
    for (int i = 0; i < half; ++i) {
      const double give = upper ? w[i] : w[half + i];
      const double keep = upper ? w[half + i] : w[i];
      w[i] = keep + __shfl_xor_sync(0xffffffffu, give, off);
    }
  }
  double mine = w[0];  // component ((lane >> (5 - L)) of the padded P)
#pragma unroll
  for (int off = 16 >> L; off > 0; off >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, off);
  constexpr int kSpan = 32 / P;  // lanes per component after the reduce-scatter
#pragma unroll
  for (int c = 0; c < K; ++c)
    y[c] = make_double2(__shfl_sync(0xffffffffu, mine, (2 * c) * kSpan),
                        __shfl_sync(0xffffffffu, mine, (2 * c + 1) * kSpan));
}

__host__ __device__ inline size_t reg_smem_bytes(size_t nt) {
  return size_t(kRegWarps) * kAsyncDepth * nt * sizeof(float2) + size_t(kRegWarps) * 4 * sizeof(double2);
}

template <int F, int K, int H>
__global__ void __launch_bounds__(kRegThreads, 3)
    project_rows_reg(const float2* __restrict__ x, float2* __restrict__ out, double* __restrict__ power,
                     size_t rows, int nt, const double2* __restrict__ vec, int mode, double inv_nt,
                     unsigned* __restrict__ flags) {
  static_assert(H == 1 || H == 2, "one or two warps per row");
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pair = warp / H, half = warp % H;
  float2* ring = reinterpret_cast<float2*>(smem) + size_t(warp) * kAsyncDepth * nt;
  // Exchange slots of a pair: [half][K] coordinates, then [half] partial power.
  double2* xch = reinterpret_cast<double2*>(smem + size_t(kRegWarps) * kAsyncDepth * nt * sizeof(float2)) +
                 size_t(pair) * 2 * 4;
  const int t0 = 32 * F * half;  // first frame of this warp's half
  double2 v[K][F];
#pragma unroll
  for (int c = 0; c < K; ++c)
#pragma unroll
    for (int f = 0; f < F; ++f) {
      const int t = t0 + lane + 32 * f;
      v[c][f] = t < nt ? vec[c * nt + t] : make_double2(0.0, 0.0);
    }
  auto pair_sync = [&]() {
    if constexpr (H == 2) asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory");
  };
  const size_t stride = size_t(gridDim.x) * (kRegWarps / H);
  size_t row = size_t(blockIdx.x) * (kRegWarps / H) + pair;
  auto issue = [&](size_t r, int slot) {
    if (r < rows) {
#pragma unroll
      for (int f = 0; f < F; ++f) {
        const int t = t0 + lane + 32 * f;
        if (t < nt) async_copy(ring + slot * nt + t, x + r * nt + t);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
#pragma unroll
  for (int d = 0; d < kAsyncDepth - 1; ++d) issue(row + d * stride, d);
  const bool subtract = mode & 1;
  bool bad_in = false, bad_out = false;
  for (int i = 0; row < rows; ++i, row += stride) {
    issue(row + (kAsyncDepth - 1) * stride, (i + kAsyncDepth - 1) % kAsyncDepth);
    asm volatile("cp.async.wait_group %0;" ::"n"(kAsyncDepth - 1) : "memory");
    const float2* cur = ring + (i % kAsyncDepth) * nt;
    double2 xv[F];
#pragma unroll
    for (int f = 0; f < F; ++f) {
      const int t = t0 + lane + 32 * f;
      if (t < nt) {
        const float2 a = cur[t];
        xv[f] = make_double2(double(a.x), double(a.y));
        bad_in |= !isfinite(a.x) || !isfinite(a.y);
      } else {
        xv[f] = make_double2(0.0, 0.0);
      }
    }
    double part[2 * K];
#pragma unroll
    for (int c = 0; c < K; ++c) {
      double yr = 0.0, yi = 0.0;
#pragma unroll
      for (int f = 0; f < F; ++f) {
        yr = fma(xv[f].x, v[c][f].x, fma(-xv[f].y, v[c][f].y, yr));
        yi = fma(xv[f].x, v[c][f].y, fma(xv[f].y, v[c][f].x, yi));
      }
      part[2 * c] = yr;
      part[2 * c + 1] = yi;
    }
    double2 y[K];
    warp_sum_coordinates<K>(part, lane, y);
    if constexpr (H == 2) {  // the pair's two halves, half 0 first
      if (lane == 0)
#pragma unroll
        for (int c = 0; c < K; ++c) xch[half * 4 + c] = y[c];
      pair_sync();
#pragma unroll
      for (int c = 0; c < K; ++c)
        y[c] = make_double2(xch[c].x + xch[4 + c].x, xch[c].y + xch[4 + c].y);
    }
    double retained = 0.0;
#pragma unroll
    for (int c = 0; c < K; ++c) retained += y[c].x * y[c].x + y[c].y * y[c].y;
    double pw = 0.0;
    if (mode & 3) {
#pragma unroll
      for (int f = 0; f < F; ++f) {
        const int t = t0 + lane + 32 * f;
        if (t < nt) {
          double2 proj = make_double2(0.0, 0.0);
#pragma unroll
          for (int c = 0; c < K; ++c) {  // y * conj(v)
            proj.x = fma(y[c].x, v[c][f].x, fma(y[c].y, v[c][f].y, proj.x));
            proj.y = fma(y[c].y, v[c][f].x, fma(-y[c].x, v[c][f].y, proj.y));
          }
          const double2 r = subtract ? make_double2(xv[f].x - proj.x, xv[f].y - proj.y) : proj;
          pw += r.x * r.x + r.y * r.y;
          if (mode & 2) out[row * nt + t] = make_float2(float(r.x), float(r.y));
        }
      }
    }
    if (power) {
      if (subtract) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) pw += __shfl_xor_sync(0xffffffffu, pw, off);
        if constexpr (H == 2) {  // slot 3 of each half holds its partial power
          if (lane == 0) xch[half * 4 + 3].x = pw;
          pair_sync();
          pw = xch[3].x + xch[4 + 3].x;
        }
      } else {
        pw = retained;
      }
      if (lane == 0 && half == 0) {
        power[row] = pw * inv_nt;
        bad_out |= !isfinite(pw);
      }
    }
    pair_sync();  // the exchange slots are read before the next row writes them
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  if (flags) {
    const unsigned bits = (__any_sync(0xffffffffu, bad_in) ? 1u : 0u) | (__any_sync(0xffffffffu, bad_out) ? 2u : 0u);
    if (bits && lane == 0) atomicOr(flags, bits);
  }
}

// Float64 tensor-core (DMMA, mma.sync m8n8k4 f64) filtered power and filtered
// IQ for complex64 rows with the smaller projector subtracted (mode 1: power;
// mode 3: the residual written to out, power optional): k <= 4 vectors,
// nt <= 512 frames.  A warp takes eight rows at a time; lane
// l works on row r = l / 4 of its group and, for every 4-frame tile j, on the
// complex sample x[r][4 j + l % 4] (one 8-byte load).  As real matrices over
// the interleaved (re, im) components:
//   Y[8 x 8]  = X[8 x 2T] W1[2T x 8]     (the k complex coordinates, padded)
//   R[8 x 2T] = X - Y W2[8 x 2T]         (the explicit residual)
// with the K dimension of the first product ordered so that step 2 j + i gives
// lane l the component i of its own sample of tile j: each loaded sample is
// the A fragment of two steps of the first product and, read again, the C
// fragment (X) of the second product's tile j.  W1 and -W2 are laid out in
// shared memory in fragment order (32 doubles per step), the coordinates move
// from the first product's D layout to the second's A layout with four
// shuffles, and each lane adds the squares of its two residual components of
// every tile.  The float64 work is the register form's (coordinates, residual,
// squares) in about a tenth of the instructions.  Samples are read in batches
// of B tiles, the next batch in flight while the current one is multiplied;
// the second read is served by L1 / L2.  8 warps per CTA share the tables;
// at most 85 registers, so three CTAs fit an SM where the tables allow.
constexpr int kDmmaMaxK = 4;

__host__ __device__ inline size_t dmma_smem_bytes(int tiles) { return size_t(tiles) * 4 * 32 * sizeof(double); }

__device__ __forceinline__ void dmma_f64(double& d0, double& d1, double a, double b, double c0, double c1) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%4, %5};"
      : "=d"(d0), "=d"(d1)
      : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

constexpr int kDmmaThreads = 256;
constexpr int kDmmaWarps = kDmmaThreads / 32;

template <int B>
__global__ void __launch_bounds__(kDmmaThreads, 3)
    project_power_dmma(const float2* __restrict__ x, float2* __restrict__ out, double* __restrict__ power,
                       size_t rows, int nt, const double2* __restrict__ vec, int k, double inv_nt,
                       unsigned* __restrict__ flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int tiles = (nt + 3) / 4;
  double* b1 = reinterpret_cast<double*>(smem);  // [2 tiles][32]: step s = 2 j + i
  double* b2 = b1 + size_t(tiles) * 2 * 32;     // [tiles][2 k-steps][32]
  // W1 (step s = 2 j + i, lane l: K row = component i of frame 4 j + l % 4,
  // N column n = l / 4 = coordinate (n / 2, re / im)):
  //   yr = sum xr vr - xi vi,  yi = sum xr vi + xi vr.
  // -W2 (tile j, k-step h, lane l: K row = coordinate component 4 h + l % 4,
  // N column n = l / 4 = component n % 2 of frame 4 j + n / 2):
  //   r.re = x.re - (yr vr + yi vi),  r.im = x.im - (yi vr - yr vi).
  for (int e = threadIdx.x; e < tiles * 2 * 32; e += blockDim.x) {
    const int s = e >> 5, l = e & 31;
    {
      const int j = s >> 1, i = s & 1, t = 4 * j + (l & 3), n = l >> 2, c = n >> 1, pt = n & 1;
      double w = 0.0;
      if (t < nt && c < k) {
        const double2 v = vec[size_t(c) * nt + t];
        w = i == 0 ? (pt == 0 ? v.x : v.y) : (pt == 0 ? -v.y : v.x);
      }
      b1[e] = w;
    }
    {
      const int j = s >> 1, h = s & 1, comp = 4 * h + (l & 3), c = comp >> 1, pc = comp & 1, n = l >> 2;
      const int t = 4 * j + (n >> 1), o = n & 1;
      double w = 0.0;
      if (t < nt && c < k) {
        const double2 v = vec[size_t(c) * nt + t];
        w = o == 0 ? (pc == 0 ? -v.x : -v.y) : (pc == 0 ? v.y : -v.x);
      }
      b2[e] = w;
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = lane & 3;
  const size_t groups = (rows + 7) / 8;
  bool bad_in = false, bad_out = false;
  for (size_t g = size_t(blockIdx.x) * kDmmaWarps + warp; g < groups;
       g += size_t(gridDim.x) * kDmmaWarps) {
    const size_t r = 8 * g + (lane >> 2);
    const bool live = r < rows;
    const float2* row = x + r * size_t(nt);
    auto load = [&](int j) {
      const int t = 4 * j + q;
      return (j < tiles && live && t < nt) ? row[t] : make_float2(0.f, 0.f);
    };
    float2 cur[B], nxt[B];
#pragma unroll
    for (int i = 0; i < B; ++i) cur[i] = load(i);
    double y[4][2] = {};
    for (int jb = 0; jb < tiles; jb += B) {
#pragma unroll
      for (int i = 0; i < B; ++i) nxt[i] = load(jb + B + i);
#pragma unroll
      for (int i = 0; i < B; ++i) {
        const int j = jb + i;
        if (j < tiles) {
          bad_in |= !isfinite(cur[i].x) || !isfinite(cur[i].y);
          dmma_f64(y[(2 * i) & 3][0], y[(2 * i) & 3][1], double(cur[i].x), b1[(2 * j) * 32 + lane],
                   y[(2 * i) & 3][0], y[(2 * i) & 3][1]);
          dmma_f64(y[(2 * i + 1) & 3][0], y[(2 * i + 1) & 3][1], double(cur[i].y), b1[(2 * j + 1) * 32 + lane],
                   y[(2 * i + 1) & 3][0], y[(2 * i + 1) & 3][1]);
        }
      }
#pragma unroll
      for (int i = 0; i < B; ++i) cur[i] = nxt[i];
    }
    // Lane l holds Y[r][2 q], Y[r][2 q + 1] (coordinate q: re, im); the A
    // fragment of k-step h of R = X - Y W2 is component 4 h + q of row r.
    const double y0 = (y[0][0] + y[1][0]) + (y[2][0] + y[3][0]);
    const double y1 = (y[0][1] + y[1][1]) + (y[2][1] + y[3][1]);
    double a[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int src = (lane & ~3) + 2 * h + (q >> 1);
      const double s0 = __shfl_sync(0xffffffffu, y0, src), s1 = __shfl_sync(0xffffffffu, y1, src);
      a[h] = (q & 1) ? s1 : s0;
    }
    double pw[2] = {0.0, 0.0};
#pragma unroll
    for (int i = 0; i < B; ++i) cur[i] = load(i);
    for (int jb = 0; jb < tiles; jb += B) {
#pragma unroll
      for (int i = 0; i < B; ++i) nxt[i] = load(jb + B + i);
#pragma unroll
      for (int i = 0; i < B; ++i) {
        const int j = jb + i;
        if (j < tiles) {
          double d0, d1;
          dmma_f64(d0, d1, a[0], b2[(2 * j) * 32 + lane], double(cur[i].x), double(cur[i].y));
          dmma_f64(d0, d1, a[1], b2[(2 * j + 1) * 32 + lane], d0, d1);
          pw[i & 1] = fma(d0, d0, fma(d1, d1, pw[i & 1]));
          if (out && live && 4 * j + q < nt) out[r * size_t(nt) + 4 * j + q] = make_float2(float(d0), float(d1));
        }
      }
#pragma unroll
      for (int i = 0; i < B; ++i) cur[i] = nxt[i];
    }
    double p = pw[0] + pw[1];
    p += __shfl_xor_sync(0xffffffffu, p, 1);
    p += __shfl_xor_sync(0xffffffffu, p, 2);
    if (power && q == 0 && live) {
      power[r] = p * inv_nt;
      bad_out |= !isfinite(p);
    }
  }
  if (flags) {
    const unsigned bits = (__any_sync(0xffffffffu, bad_in) ? 1u : 0u) | (__any_sync(0xffffffffu, bad_out) ? 2u : 0u);
    if (bits && lane == 0) atomicOr(flags, bits);
  }
}

// The flags of project_rows_async for the other projection kernels: bit 0 for
// a non-finite input component, bit 1 for a non-finite power (when given).
template <typename IN>
__global__ void input_flags(const IN* __restrict__ x, size_t n, unsigned* __restrict__ flags) {
  bool bad = false;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    bad |= !isfinite(double(x[i].x)) || !isfinite(double(x[i].y));
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flags, 1u);
}

__global__ void power_flags(const double* __restrict__ power, size_t rows, unsigned* __restrict__ flags) {
  bool bad = false;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < rows; i += size_t(gridDim.x) * blockDim.x)
    bad |= !isfinite(power[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flags, 2u);
}

constexpr int kRefineRows = 16;  // Casorati rows staged per block of the Rayleigh-Ritz pass

// Float64 Rayleigh-Ritz matrix of the Casorati rows on m <= kRitzMax vectors:
// h (m x m complex128, column-major, accumulated with atomics) += Y^H Y with
// Y = X V, i.e. V^H G V for the exact Gram G = X^H X, without forming G.  Per
// CTA, blocks of kRefineRows rows are staged in shared memory; thread (row, c)
// forms y[row][c] over all frames, then thread (i, j) accumulates
// conj(y[r][i]) y[r][j] over the block's rows in a register.  V's rows are
// staged with a padded stride so that the 16 vectors a warp reads sit in
// distinct banks.
constexpr int kRitzMax = 16;
constexpr int kRitzThreads = kRefineRows * kRitzMax;  // 256

__host__ __device__ inline int ritz_stride(int nt) { return nt + 1; }  // double2 elements per staged vector

__global__ void __launch_bounds__(kRitzThreads)
    ritz_matrix(const float2* __restrict__ x, size_t rows, int nt, const double2* __restrict__ vec, int m,
                double* __restrict__ h) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int vs_stride = ritz_stride(nt);
  double2* vs = reinterpret_cast<double2*>(smem);                        // [m][nt + 1]
  double2* ys = vs + size_t(kRitzMax) * vs_stride;                       // [rows][kRitzMax]
  float2* xs = reinterpret_cast<float2*>(ys + kRefineRows * kRitzMax);   // [rows][nt]
  for (int i = threadIdx.x; i < m * nt; i += blockDim.x) vs[(i / nt) * vs_stride + i % nt] = vec[i];
  const size_t per = (rows + gridDim.x - 1) / gridDim.x;
  const size_t r0 = size_t(blockIdx.x) * per, r1 = min(rows, r0 + per);
  const int pr = threadIdx.x / kRitzMax, pc = threadIdx.x % kRitzMax;  // (row, vector) of phase 1
  const int hi = threadIdx.x / kRitzMax, hj = threadIdx.x % kRitzMax;  // (i, j) of phase 2
  double hr = 0.0, him = 0.0;
  for (size_t b = r0; b < r1; b += kRefineRows) {
    const int nr = int(min(size_t(kRefineRows), r1 - b));
    __syncthreads();
    for (int i = threadIdx.x; i < nr * nt; i += blockDim.x) xs[i] = x[b * size_t(nt) + i];
    __syncthreads();
    double yr = 0.0, yi = 0.0;
    if (pr < nr && pc < m) {
      const float2* xr = xs + pr * nt;
      const double2* vr = vs + pc * vs_stride;
      for (int t = 0; t < nt; ++t) {
        const float2 a = xr[t];
        const double2 v = vr[t];
        yr = fma(double(a.x), v.x, fma(-double(a.y), v.y, yr));
        yi = fma(double(a.x), v.y, fma(double(a.y), v.x, yi));
      }
    }
    ys[pr * kRitzMax + pc] = make_double2(yr, yi);
    __syncthreads();
    if (hi < m && hj < m) {
      for (int r = 0; r < nr; ++r) {
        const double2 a = ys[r * kRitzMax + hi], c = ys[r * kRitzMax + hj];
        hr = fma(a.x, c.x, fma(a.y, c.y, hr));   // conj(a) c
        him = fma(a.x, c.y, fma(-a.y, c.x, him));
      }
    }
  }
  if (hi < m && hj < m) {
    atomicAdd(h + 2 * (size_t(hj) * m + hi), hr);  // column-major (i, j)
    atomicAdd(h + 2 * (size_t(hj) * m + hi) + 1, him);
  }
}

}  // namespace clutter
}  // namespace rcb
