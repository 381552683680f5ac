// rcabeam C ABI for B200 (sm_100a).  One translation unit: every kernel of the
// library is included here so that the device error word is a single object.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cub/device/device_radix_sort.cuh>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include <cusolverDn.h>

#include "clutter.cuh"
#include "common.cuh"
#include "batch.cuh"
#include "das_adjoint.cuh"
#include "das_generic.cuh"
#include "das_staged.cuh"
#include "das_tc.cuh"
#include "gram_tc.cuh"
#include "pack.cuh"
#include "scene.cuh"

namespace rcb {

// Device error word written by bounded waits that gave up.
__device__ int g_device_error = 0;

static int* device_error_ptr() {
  int* p = nullptr;
  if (cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_device_error) != cudaSuccess) return nullptr;
  return p;
}

// ------------------------------------------------------------ TMA maps --
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Packed (slabs = nc * na, ns, nt) ensemble as a 3-D tensor of elem_bytes elements.
static bool make_slab_map(CUtensorMap* map, const void* base, int elem_bytes, size_t nt, size_t ns, size_t slabs,
                          int box_frames, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {nt, ns, slabs};
  cuuint64_t strides[2] = {nt * elem_bytes, nt * ns * elem_bytes};
  cuuint32_t box[3] = {cuuint32_t(box_frames), cuuint32_t(box_rows), 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUtensorMapDataType dt = elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32;
  return fn(map, dt, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Packed 16-bit (re, im) plane (slabs, ns, 2 nt) as 16-bit elements with 64 x 16
// SWIZZLE_128B boxes: the MN-major tensor-core operand layout.
static bool make_plane_map(CUtensorMap* map, const void* base, size_t nt, size_t ns, size_t slabs) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {2 * nt, ns, slabs};
  cuuint64_t strides[2] = {2 * nt * 2, 2 * nt * 2 * ns};
  cuuint32_t box[3] = {cuuint32_t(tc::kBoxCols), cuuint32_t(tc::kRows), 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// -------------------------------------------------- voxel traversal order --
// Morton (Z-order) codes of isotropically quantized voxel positions, sorted
// with a radix sort, give tiles of 64 consecutive voxels that are compact in
// space -- which keeps each tile's sample window short.  Uses the caller's
// geometry workspace as scratch; returns nullptr (identity order) when the
// call is small or the scratch does not fit.
__device__ __forceinline__ unsigned ordered_bits(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void bbox_kernel(const float* scan, size_t nv, unsigned* box) {
  unsigned lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nv; i += size_t(gridDim.x) * blockDim.x) {
    for (int d = 0; d < 3; ++d) {
      unsigned u = ordered_bits(scan[3 * i + d]);
      lo[d] = min(lo[d], u);
      hi[d] = max(hi[d], u);
    }
  }
  for (int d = 0; d < 3; ++d) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[d] = min(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], off));
      hi[d] = max(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], off));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(box + d, lo[d]);
      atomicMax(box + 3 + d, hi[d]);
    }
  }
}

__device__ __forceinline__ unsigned spread10(unsigned x) {
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__global__ void morton_kernel(const float* scan, size_t nv, const unsigned* box, unsigned* keys, unsigned* vals) {
  size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  float lo[3], extent = 0.f;
  for (int d = 0; d < 3; ++d) {
    lo[d] = from_ordered(box[d]);
    extent = fmaxf(extent, from_ordered(box[3 + d]) - lo[d]);
  }
  float scale = extent > 0.f ? 1023.f / extent : 0.f;
  unsigned q[3];
  for (int d = 0; d < 3; ++d) {
    float t = (scan[3 * i + d] - lo[d]) * scale + 0.5f;
    q[d] = unsigned(fminf(fmaxf(t, 0.f), 1023.f));
  }
  // z (depth) is the slowest-varying bit of each triple so that lateral
  // neighbours group first; depth moves the delay fastest.
  keys[i] = (spread10(q[1]) << 2) | (spread10(q[0]) << 1) | spread10(q[2]);
  vals[i] = unsigned(i);
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Scratch bytes of voxel_order for nv voxels (0 when no order is built).
static size_t order_bytes(size_t nv, size_t* temp_bytes) {
  if (nv < 2 * das::kTileVoxels || nv > 0x7fffffffull) return 0;
  cub::DoubleBuffer<unsigned> keys(nullptr, nullptr), vals(nullptr, nullptr);
  size_t temp = 0;
  if (cub::DeviceRadixSort::SortPairs(nullptr, temp, keys, vals, int(nv), 0, 30, cudaStream_t(0)) != cudaSuccess)
    return 0;
  if (temp_bytes) *temp_bytes = temp;
  return 4 * align256(nv * 4) + 256 + align256(temp);
}

static const unsigned* voxel_order(const float* scan, size_t nv, void* workspace, size_t workspace_bytes) {
  size_t temp = 0;
  size_t need = order_bytes(nv, &temp);
  if (!need || need > workspace_bytes) return nullptr;
  size_t n4 = align256(nv * 4);
  cub::DoubleBuffer<unsigned> keys(nullptr, nullptr), vals(nullptr, nullptr);
  unsigned char* w = static_cast<unsigned char*>(workspace);
  unsigned* ka = reinterpret_cast<unsigned*>(w);
  unsigned* kb = reinterpret_cast<unsigned*>(w + n4);
  unsigned* va = reinterpret_cast<unsigned*>(w + 2 * n4);
  unsigned* vb = reinterpret_cast<unsigned*>(w + 3 * n4);
  unsigned* box = reinterpret_cast<unsigned*>(w + 4 * n4);
  void* tmp = w + 4 * n4 + 256;
  // 0xff.. bytes for the three minima, zero bytes for the three maxima.
  if (cudaMemsetAsync(box, 0xff, 12, 0) != cudaSuccess || cudaMemsetAsync(box + 3, 0, 12, 0) != cudaSuccess)
    return nullptr;
  bbox_kernel<<<148, 256>>>(scan, nv, box);
  morton_kernel<<<unsigned((nv + 255) / 256), 256>>>(scan, nv, box, ka, va);
  keys = cub::DoubleBuffer<unsigned>(ka, kb);
  vals = cub::DoubleBuffer<unsigned>(va, vb);
  if (cub::DeviceRadixSort::SortPairs(tmp, temp, keys, vals, int(nv), 0, 30, cudaStream_t(0)) != cudaSuccess)
    return nullptr;
  if (cudaGetLastError() != cudaSuccess) return nullptr;
  return vals.Current();
}

// ---------------------------------------------------------- dispatch --
static unsigned pow2_at_least(unsigned x) {
  unsigned p = 1;
  while (p < x) p <<= 1;
  return p;
}

template <int LPV, bool HALF, int MODE, bool TMA>
static rcabeam_status launch_staged(const CUtensorMap& mr, const CUtensorMap& mq, const das::Args& a, dim3 grid,
                                    cudaStream_t stream) {
  using S = das::Shape<LPV, HALF>;
  auto kern = das::opw_staged<LPV, HALF, MODE, TMA>;
  size_t smem = S::bytes(a.na);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  kern<<<grid, das::kThreads, smem, stream>>>(mr, mq, a);
  return launch_status();
}

template <bool HALF, int MODE, bool TMA>
static rcabeam_status launch_lpv(int lpv, const CUtensorMap& mr, const CUtensorMap& mq, const das::Args& a,
                                 dim3 grid, cudaStream_t stream) {
  switch (lpv) {
    case 32: return launch_staged<32, HALF, MODE, TMA>(mr, mq, a, grid, stream);
    case 16: return launch_staged<16, HALF, MODE, TMA>(mr, mq, a, grid, stream);
    case 8: return launch_staged<8, HALF, MODE, TMA>(mr, mq, a, grid, stream);
    case 4: return launch_staged<4, HALF, MODE, TMA>(mr, mq, a, grid, stream);
    default: return launch_staged<2, HALF, MODE, TMA>(mr, mq, a, grid, stream);
  }
}

template <bool HALF, int MODE>
static rcabeam_status run_staged(das::Args a, size_t ntiles, cudaStream_t stream = 0) {
  const int elem = HALF ? 4 : 8;
  const size_t nt = size_t(a.nt);
  const bool aligned = (nt * elem) % 16 == 0 && reinterpret_cast<uintptr_t>(a.rc) % 16 == 0 &&
                       reinterpret_cast<uintptr_t>(a.cr) % 16 == 0 && encode_fn() != nullptr;
  const int main_chunks = int(nt / 64);
  const int tail = int(nt % 64);
  struct Launch {
    int lpv, frames, chunks, base;
  } launches[2];
  int count = 0;
  if (main_chunks) launches[count++] = {32, 64, main_chunks, 0};
  if (tail) {
    int frames = int(pow2_at_least(unsigned(tail)));
    if (frames < 4) frames = 4;
    launches[count++] = {frames / 2, frames, 1, main_chunks * 64};
  }
  for (int i = 0; i < count; ++i) {
    CUtensorMap mr{}, mq{};
    bool tma = aligned && make_slab_map(&mr, a.rc, elem, nt, size_t(a.ns), size_t(a.nc) * a.na,
                                        launches[i].frames, das::kRows) &&
               make_slab_map(&mq, a.cr, elem, nt, size_t(a.ns), size_t(a.nc) * a.na, launches[i].frames, das::kRows);
    das::Args b = a;
    b.frame_base = launches[i].base;
    dim3 grid(unsigned(ntiles), unsigned(launches[i].chunks));
    rcabeam_status st = tma ? launch_lpv<HALF, MODE, true>(launches[i].lpv, mr, mq, b, grid, stream)
                            : launch_lpv<HALF, MODE, false>(launches[i].lpv, mr, mq, b, grid, stream);
    if (st != RCABEAM_SUCCESS) return st;
  }
  return RCABEAM_SUCCESS;
}

// DMAS-CCF-ACF on the staged pipeline: 32-frame chunks, both passes per CTA.
static rcabeam_status run_dmas_staged(das::Args a, size_t ntiles, cudaStream_t stream = 0) {
  constexpr int kLpv = 16;
  using S = das::Shape<kLpv, false>;
  const size_t nt = size_t(a.nt);
  const bool aligned = (nt * 8) % 16 == 0 && reinterpret_cast<uintptr_t>(a.rc) % 16 == 0 &&
                       reinterpret_cast<uintptr_t>(a.cr) % 16 == 0 && encode_fn() != nullptr;
  CUtensorMap mr{}, mq{};
  const size_t slabs = size_t(a.nc) * a.na;
  const bool tma = aligned && make_slab_map(&mr, a.rc, 8, nt, size_t(a.ns), slabs, S::kFrames, das::kRows) &&
                   make_slab_map(&mq, a.cr, 8, nt, size_t(a.ns), slabs, S::kFrames, das::kRows);
  const dim3 grid(unsigned(ntiles), unsigned((nt + S::kFrames - 1) / S::kFrames));
  const size_t smem = S::bytes(a.na);
  auto kern = tma ? das::dmas_staged<kLpv, true> : das::dmas_staged<kLpv, false>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  kern<<<grid, das::kThreads, smem, stream>>>(mr, mq, a);
  return launch_status();
}

static bool tc_eligible(const void* const* planes, int count, size_t nt) {
  if (nt % 4 != 0 || !encode_fn()) return false;
  for (int i = 0; i < count; ++i)
    if (!planes[i] || reinterpret_cast<uintptr_t>(planes[i]) % 16 != 0) return false;
  return true;
}

// Shared memory of the tensor-core OPW for nt frames and na angles (0 if it cannot run).
// Shared memory of the tensor-core kernel with `stages` ring stages (0: does not fit).
// Frame passes of the tensor-core OPW: full passes of 128 frames (N = 256, four
// whole 64-column boxes per plane) and a last pass with the remainder rounded up
// to 8 frames, which stages fewer boxes than equal passes would.
// Frames of every frame pass but the last: passes of nearly equal length
// (multiples of 8 frames, at most kMaxFrames).  Equal passes keep the CTAs'
// items equally long, so the herd's channel walks stay aligned (200 frames:
// 104 + 96 ran the DAS 2.5 % faster than 128 + 72).
static size_t tc_full_frames(size_t nt) {
  if (nt <= size_t(tc::kMaxFrames)) return (nt + 7) / 8 * 8;
  const size_t passes = (nt + tc::kMaxFrames - 1) / tc::kMaxFrames;
  return ((nt + passes - 1) / passes + 7) / 8 * 8;
}

static size_t tc_smem_bytes(bool bf16x3, size_t nt, size_t na, int stages = tc::kStages) {
  const size_t frames = tc_full_frames(nt);
  const int nbox = int((2 * frames + tc::kBoxCols - 1) / tc::kBoxCols);
  size_t smem = (bf16x3 ? tc::Layout<true>::bytes(nbox, int(na), stages)
                        : tc::Layout<false>::bytes(nbox, int(na), stages)) + 1024;
  if (smem < 120 * 1024) smem = 120 * 1024;  // one CTA per SM: each owns all 512 TMEM columns
  return smem <= 227 * 1024 ? smem : 0;
}

// Tensor-core OPW over all (tile, frame pass) work items with one persistent CTA per SM.
// Segment sums of the tensor-core DAS (one slice per resident CTA; launches
// are serialized on the default stream, so one buffer per device suffices).
static __device__ float2 g_tc_partials[tc::kMaxCtas * tc::kPartialPerCta];
// Work-item counter of the tensor-core DAS (one launch at a time per device,
// like the segment scratch above).
static __device__ unsigned g_tc_items;

// Global channel-slot count of the tensor-core DAS (its phase aligns the CTAs'
// slab walks; any starting value works, so it is never reset).
static __device__ unsigned long long g_tc_slot_clock;

static unsigned long long* tc_slot_clock_address() {
  static std::mutex lock;
  static unsigned long long* addresses[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> guard(lock);
  if (!addresses[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_tc_slot_clock) != cudaSuccess) return nullptr;
    addresses[dev] = static_cast<unsigned long long*>(ptr);
  }
  return addresses[dev];
}

static float2* tc_partials_address() {
  static std::mutex lock;
  static float2* addresses[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> guard(lock);
  if (!addresses[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_tc_partials) != cudaSuccess) return nullptr;
    addresses[dev] = static_cast<float2*>(ptr);
  }
  return addresses[dev];
}

// MMA steps per float32 accumulation segment (RCABEAM_TC_SEGMENT overrides, for a/b runs).
static int segment_steps() {
  const char* v = std::getenv("RCABEAM_TC_SEGMENT");
  const int n = v ? std::atoi(v) : 0;
  return n >= 16 && n <= 4096 ? n : tc::kSegSteps;
}

template <bool BF16X3>
static rcabeam_status run_tc(tc::Args a) {
  a.seg_steps = segment_steps();
  const size_t nt = size_t(a.nt);
  // The deepest ring (one builder warp per stage) that fits shared memory.
  int stages = tc::kDeepStages;
  size_t smem = 0;
  for (; stages >= 2; --stages)
    if ((smem = tc_smem_bytes(BF16X3, nt, size_t(a.na), stages))) break;
  if (!smem) return RCABEAM_ERROR_ARGUMENT;
  a.chunks = int((nt + tc::kMaxFrames - 1) / tc::kMaxFrames);
  const int frames = int(tc_full_frames(nt));
  a.frames = frames;
  a.last_frames = int((nt - size_t(frames) * size_t(a.chunks - 1) + 7) / 8 * 8);
  a.ncols = 2 * frames;
  a.nbox = (a.ncols + tc::kBoxCols - 1) / tc::kBoxCols;
  a.ntiles = int((size_t(a.nv) + tc::kVox - 1) / tc::kVox);
  CUtensorMap mh[2], ml[2];
  const size_t slabs = size_t(a.nc) * a.na;
  for (int i = 0; i < 2; ++i) {
    if (!make_plane_map(&mh[i], a.x_hi[i], nt, size_t(a.ns), slabs)) return RCABEAM_ERROR_CUDA;
    if (BF16X3) {
      if (!make_plane_map(&ml[i], a.x_lo[i], nt, size_t(a.ns), slabs)) return RCABEAM_ERROR_CUDA;
    } else {
      ml[i] = mh[i];
    }
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto kern = stages == 6   ? tc::opw_tc<BF16X3, 6>
              : stages == 5 ? tc::opw_tc<BF16X3, 5>
              : stages == 4 ? tc::opw_tc<BF16X3, 4>
              : stages == 3 ? tc::opw_tc<BF16X3, 3>
                            : tc::opw_tc<BF16X3, 2>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  a.partial = tc_partials_address();
  a.slot_clock = tc_slot_clock_address();
  if (!a.partial || !a.slot_clock) return RCABEAM_ERROR_CUDA;
  const int items = a.ntiles * a.chunks;
  const unsigned grid = unsigned(std::min(std::min(items, sms), tc::kMaxCtas));
  // CTAs take work items from a counter (zeroed here, on the launch's stream):
  // DAS 826 -> 803 ms at the full-size workload against the static b, b + G, ...
  void* counter = nullptr;
  if (cudaGetSymbolAddress(&counter, g_tc_items) != cudaSuccess ||
      cudaMemsetAsync(counter, 0, sizeof(unsigned), 0) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  a.item_counter = static_cast<unsigned*>(counter);
  kern<<<grid, tc::threads_for(stages), smem>>>(mh[0], mh[1], ml[0], ml[1], a);
  return launch_status();
}

template <bool HALF>
static rcabeam_status ensemble_impl(const void* rc, const void* cr, const float* scan, const float* xe,
                                    const float* ye, const float* angles, const float* starts, float* pd,
                                    void* signal, float* weights, void* workspace, void* geometry_workspace, size_t ns,
                                    size_t nc, size_t na, size_t nt, size_t nv, float c, float fs, float fd, float fn,
                                    int method, int k) {
  // Argument contract of the reference (ensemble.cu:664-675).
  if (!rc || !cr || !scan || !xe || !ye || !angles || !starts || !pd || ns < 2 || !nc || !na || !nt || !nv ||
      c <= 0 || fs <= 0 || method < 0 || method > 5 || (method == 5 && !signal) || !std::isfinite(c) ||
      !std::isfinite(fs) || !std::isfinite(fd) || !std::isfinite(fn))
    return RCABEAM_ERROR_ARGUMENT;
  if (HALF && method != 0) return RCABEAM_ERROR_ARGUMENT;
  if (method == 4 && (!weights || !workspace || signal || k < 2 || k > 4 || na < size_t(k)))
    return RCABEAM_ERROR_ARGUMENT;
  if (!geometry_workspace) return RCABEAM_ERROR_ARGUMENT;
  // Index ranges of the kernels (32-bit sample, channel, angle, frame and voxel ids).
  if (ns > INT32_MAX || nc > INT32_MAX || na > INT32_MAX || nt > INT32_MAX || nv > INT32_MAX ||
      nc * na > INT32_MAX || na > 4096)
    return RCABEAM_ERROR_ARGUMENT;
  if (cudaMemsetAsync(pd, 0, 2 * nv * sizeof(float), 0) != cudaSuccess) return RCABEAM_ERROR_CUDA;
  das::Args a{};
  a.rc = rc;
  a.cr = cr;
  a.scan = scan;
  a.xe = xe;
  a.ye = ye;
  a.angles = angles;
  a.starts = starts;
  a.pd = pd;
  a.signal = static_cast<float2*>(signal);
  a.ns = int(ns);
  a.nc = int(nc);
  a.na = int(na);
  a.nt = int(nt);
  a.nv = int(nv);
  a.c = double(c);
  a.fs = double(fs);
  a.fd = double(fd);
  a.fn = double(fn);
  a.err = device_error_ptr();
  if (method == 2) {
    dim3 grid(unsigned((nv + generic::kWarps - 1) / generic::kWarps),
              unsigned((nt + 32 * generic::kRegFrames - 1) / (32 * generic::kRegFrames)));
    generic::ensemble_nonlinear<2><<<grid, generic::kWarps * 32>>>(a);
    return launch_status();
  }
  if (method == 4) {
    // St-SW: series into the caller's workspace (nv k^2 nt complex64), then
    // energies, pair sums, raw weights and the XDoppler magnitude.
    constexpr int kStswFrames = generic::kRegFrames;
    const unsigned blocks = unsigned((nv + generic::kWarps - 1) / generic::kWarps);
    dim3 grid(blocks, unsigned((nt + 32 * kStswFrames - 1) / (32 * kStswFrames)));
    float2* series = static_cast<float2*>(workspace);
    if (k == 2) {
      generic::stsw_series<2, kStswFrames><<<grid, generic::kWarps * 32>>>(a, series);
      generic::stsw_finish<2><<<blocks, generic::kWarps * 32>>>(pd, weights, series, nv, int(nt));
    } else if (k == 3) {
      generic::stsw_series<3, kStswFrames><<<grid, generic::kWarps * 32>>>(a, series);
      generic::stsw_finish<3><<<blocks, generic::kWarps * 32>>>(pd, weights, series, nv, int(nt));
    } else {
      generic::stsw_series<4, kStswFrames><<<grid, generic::kWarps * 32>>>(a, series);
      generic::stsw_finish<4><<<blocks, generic::kWarps * 32>>>(pd, weights, series, nv, int(nt));
    }
    return launch_status();
  }
  // The caller owns 2 * nv * (nc + na) float4 of scratch (reference rcabeam.h:196).
  a.order = voxel_order(scan, nv, geometry_workspace, 2 * nv * (nc + na) * 16);
  if (method == 3) return run_dmas_staged(a, (nv + das::kTileVoxels - 1) / das::kTileVoxels);
  const size_t ntiles = (nv + das::kTileVoxels - 1) / das::kTileVoxels;
  const void* planes[2] = {rc, cr};
  if (HALF && tc_eligible(planes, 2, nt) && nv <= size_t(INT32_MAX) - tc::kVox && tc_smem_bytes(false, nt, na, 2)) {
    tc::Args t{};
    t.x_hi[0] = rc;
    t.x_hi[1] = cr;
    t.scan = scan;
    t.xe = xe;
    t.ye = ye;
    t.angles = angles;
    t.starts = starts;
    t.order = a.order;
    t.pd = pd;
    t.signal = a.signal;
    t.ns = a.ns;
    t.nc = a.nc;
    t.na = a.na;
    t.nt = a.nt;
    t.nv = a.nv;
    t.c = a.c;
    t.fs = a.fs;
    t.fd = a.fd;
    t.fn = a.fn;
    t.err = a.err;
    return run_tc<false>(t);
  }
  rcabeam_status st;
  if (method == 0)
    st = run_staged<HALF, das::kOpw>(a, ntiles);
  else if (method == 5)
    st = run_staged<false, das::kApertures>(a, ntiles);
  else
    st = run_staged<false, das::kXdoppler>(a, ntiles);
  if (st != RCABEAM_SUCCESS) return st;
  if (method == 1) {
    das::finish_magnitude<<<unsigned((nv + 255) / 256), 256>>>(pd, nv);
    return launch_status();
  }
  return RCABEAM_SUCCESS;
}

static generic::FrameArgs frame_args(const void* rc, const void* cr, const float* scan, const float* xe,
                                     const float* ye, const float* angles, const float* starts, size_t ns, size_t nc,
                                     size_t na, size_t nv, float c, float fs, float fd, float fn) {
  generic::FrameArgs f{};
  f.rc = static_cast<const float2*>(rc);
  f.cr = static_cast<const float2*>(cr);
  f.scan = scan;
  f.xe = xe;
  f.ye = ye;
  f.angles = angles;
  f.starts = starts;
  f.ns = int(ns);
  f.nc = int(nc);
  f.na = int(na);
  f.nv = nv;
  f.c = c;
  f.fs = fs;
  f.fd = fd;
  f.fn = fn;
  return f;
}

static bool bad_frame_args(const void* iq, const float* scan, const float* el, const float* angles,
                           const float* starts, const void* out, size_t ns, size_t nc, size_t na, size_t nv,
                           int config) {
  return !iq || !scan || !el || !angles || !starts || !out || ns < 2 || !nc || !na || !nv ||
         (config != 0 && config != 1) || ns > INT32_MAX || nc > INT32_MAX || na > INT32_MAX;
}

static unsigned blocks_for(size_t n, unsigned threads) { return unsigned((n + threads - 1) / threads); }

// One cuSOLVER handle per device, bound to the legacy default stream.
static cusolverDnHandle_t solver_handle() {
  static std::mutex lock;
  static cusolverDnHandle_t handles[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> guard(lock);
  if (!handles[dev]) {
    if (cusolverDnCreate(&handles[dev]) != CUSOLVER_STATUS_SUCCESS) return nullptr;
    cusolverDnSetStream(handles[dev], 0);
  }
  return handles[dev];
}

template <typename IN, int MAXF>
static void launch_project(const void* iq, void* out, double* power, size_t rows, size_t nt, const double* vec,
                           size_t k, int mode) {
  if (k <= size_t(clutter::kProjSmall))
    clutter::project_rows_one<IN, MAXF><<<blocks_for(rows * 32, 128), 128>>>(
        static_cast<const IN*>(iq), static_cast<IN*>(out), power, rows, int(nt),
        reinterpret_cast<const double2*>(vec), int(k), mode, 1.0 / double(nt));
  else
    clutter::project_rows<IN, MAXF><<<blocks_for(rows * 32, 256), 256>>>(
        static_cast<const IN*>(iq), static_cast<IN*>(out), power, rows, int(nt),
        reinterpret_cast<const double2*>(vec), int(k), mode, 1.0 / double(nt));
}

template <typename IN, int MAXF>
static bool launch_async(const void* iq, void* out, double* power, size_t rows, size_t nt, const double* vec,
                         size_t k, int mode, unsigned* flags) {
  auto kern = clutter::project_rows_async<IN, MAXF>;
  const size_t smem = clutter::async_smem_bytes(k, nt, sizeof(IN));
  if (smem > 110 * 1024) return false;  // keep two CTAs per SM
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return false;
  int dev = 0, sms = 148, per_sm = 2;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, clutter::kAsyncThreads, smem);
  const size_t want = (rows + clutter::kAsyncWarps - 1) / clutter::kAsyncWarps;
  const size_t grid = std::min(want, size_t(sms) * size_t(per_sm > 0 ? per_sm : 1));
  kern<<<unsigned(grid), clutter::kAsyncThreads, smem>>>(static_cast<const IN*>(iq), static_cast<IN*>(out), power,
                                                          rows, int(nt), reinterpret_cast<const double2*>(vec),
                                                          int(k), mode, 1.0 / double(nt), flags);
  return true;
}

template <int F, int K, int H>
static void launch_reg(const void* iq, void* out, double* power, size_t rows, size_t nt, const double* vec,
                       int mode, unsigned* flags) {
  auto kern = clutter::project_rows_reg<F, K, H>;
  const size_t smem = clutter::reg_smem_bytes(nt);
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  int dev = 0, sms = 148, per_sm = 3;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, clutter::kRegThreads, smem);
  const size_t rows_per_block = clutter::kRegWarps / H;
  const size_t want = (rows + rows_per_block - 1) / rows_per_block;
  const size_t grid = std::min(want, size_t(sms) * size_t(per_sm > 0 ? per_sm : 1));
  kern<<<unsigned(grid), clutter::kRegThreads, smem>>>(static_cast<const float2*>(iq), static_cast<float2*>(out),
                                                        power, rows, int(nt), reinterpret_cast<const double2*>(vec),
                                                        mode, 1.0 / double(nt), flags);
}

static void launch_dmma(const void* iq, void* out, double* power, size_t rows, size_t nt, const double* vec,
                        size_t k, unsigned* flags) {
  auto kern = clutter::project_power_dmma<8>;
  const size_t smem = clutter::dmma_smem_bytes(int((nt + 3) / 4));
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  int dev = 0, sms = 148, per_sm = 2;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, clutter::kDmmaThreads, smem);
  const size_t groups = (rows + 7) / 8;
  const size_t want = (groups + clutter::kDmmaWarps - 1) / clutter::kDmmaWarps;
  const size_t grid = std::min(want, size_t(sms) * size_t(per_sm > 0 ? per_sm : 1));
  kern<<<unsigned(grid), clutter::kDmmaThreads, smem>>>(static_cast<const float2*>(iq), static_cast<float2*>(out),
                                                         power, rows, int(nt),
                                                         reinterpret_cast<const double2*>(vec), int(k),
                                                         1.0 / double(nt), flags);
}

// Complex64 rows with the smaller projector subtracted, 1-4 vectors, 33-512
// frames: the float64 tensor-core form (mode 1: filtered power; mode 3: the
// filtered IQ, power optional).
static bool project_dmma(const void* iq, void* out, double* power, size_t rows, size_t nt, const double* vec,
                         size_t k, int mode, unsigned* flags) {
  const bool power_only = mode == 1 && power, residual = mode == 3 && out;
  if (!(power_only || residual) || k < 1 || k > size_t(clutter::kDmmaMaxK) || nt <= 32 || nt > 512) return false;
  launch_dmma(iq, residual ? out : nullptr, power, rows, nt, vec, k, flags);
  return true;
}

// Complex64, 1-3 vectors, 33-512 frames: the register form (a warp pair per
// row above 256 frames).
static bool project_reg(const void* iq, void* out, double* power, size_t rows, size_t nt, const double* vec,
                        size_t k, int mode, unsigned* flags) {
  if (k < 1 || k > 3 || nt <= 32 || nt > 512) return false;
  const int f = int((nt + 31) / 32);
  using Launch = void (*)(const void*, void*, double*, size_t, size_t, const double*, int, unsigned*);
  static const Launch table[3][4] = {  // [k - 1][F = 4, 7, 8 on one warp; 8 on a warp pair]
      {launch_reg<4, 1, 1>, launch_reg<7, 1, 1>, launch_reg<8, 1, 1>, launch_reg<8, 1, 2>},
      {launch_reg<4, 2, 1>, launch_reg<7, 2, 1>, launch_reg<8, 2, 1>, launch_reg<8, 2, 2>},
      {launch_reg<4, 3, 1>, launch_reg<7, 3, 1>, launch_reg<8, 3, 1>, launch_reg<8, 3, 2>},
  };
  table[k - 1][f <= 4 ? 0 : f <= 7 ? 1 : f <= 8 ? 2 : 3](iq, out, power, rows, nt, vec, mode, flags);
  return true;
}

template <typename IN>
static void project_dispatch(const void* iq, void* out, double* power, size_t rows, size_t nt, const double* vec,
                             size_t k, int mode, unsigned* flags) {
  if constexpr (sizeof(IN) == 8) {
    if (project_dmma(iq, out, power, rows, nt, vec, k, mode, flags)) return;
    if (project_reg(iq, out, power, rows, nt, vec, k, mode, flags)) return;
  }
  if (k <= size_t(clutter::kProjSmall)) {
    if (nt <= 256 && launch_async<IN, 8>(iq, out, power, rows, nt, vec, k, mode, flags)) return;
    if (nt > 256 && launch_async<IN, 16>(iq, out, power, rows, nt, vec, k, mode, flags)) return;
  }
  if (flags) clutter::input_flags<IN><<<296, 256>>>(static_cast<const IN*>(iq), rows * nt, flags);
  size_t f = (nt + 31) / 32;
  if (f <= 1) launch_project<IN, 1>(iq, out, power, rows, nt, vec, k, mode);
  else if (f <= 2) launch_project<IN, 2>(iq, out, power, rows, nt, vec, k, mode);
  else if (f <= 4) launch_project<IN, 4>(iq, out, power, rows, nt, vec, k, mode);
  else if (f <= 8) launch_project<IN, 8>(iq, out, power, rows, nt, vec, k, mode);
  else launch_project<IN, 16>(iq, out, power, rows, nt, vec, k, mode);
  if (flags && power) clutter::power_flags<<<148, 256>>>(power, rows, flags);
}

// ---------------------------------------------- no-allocation entry point --
// Some callers cannot call cudaMalloc at all: real-time acquisition loops whose
// device memory budget is fixed when the scanner starts (an allocation can
// synchronize the device and stall the loop for an unbounded time), and
// plugins inside host applications whose device memory belongs to another
// runtime's allocator.  For them rcabeam_ensemble_static_device keeps its
// scratch (the voxel traversal-order sort: keys, values, bounding box and
// radix-sort temporaries) in this file-scope device array instead of a
// caller-provided workspace.  Every GPU that loads the library holds the array
// until the process exits, and every call on a device shares it.
constexpr size_t kStaticMaxVoxels = size_t(1) << 18;       // 262144 voxels per call
constexpr size_t kStaticScratchBytes = size_t(8) << 20;    // 8 MiB per device
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch for the current device.  The host-side
// symbol is only a stand-in, so the address is looked up once per device with
// that device current (the first call on each device does this; make that
// first call before any stream capture).
static void* static_scratch_address() {
  static std::mutex lock;
  static void* addresses[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> guard(lock);
  if (!addresses[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_static_scratch) != cudaSuccess) return nullptr;
    addresses[dev] = ptr;
  }
  return addresses[dev];
}

static rcabeam_status ensemble_static(const void* rc, const void* cr, const float* scan, const float* xe,
                                      const float* ye, const float* angles, const float* starts, float* pd,
                                      void* signal, size_t ns, size_t nc, size_t na, size_t nt, size_t nv, float c,
                                      float fs, float fd, float fn, int method) {
  if (!rc || !cr || !scan || !xe || !ye || !angles || !starts || !pd || ns < 2 || !nc || !na || !nt || !nv ||
      c <= 0 || fs <= 0 || !std::isfinite(c) || !std::isfinite(fs) || !std::isfinite(fd) || !std::isfinite(fn))
    return RCABEAM_ERROR_ARGUMENT;
  if (method < 0 || method > 5 || method == 4 || (method == 5 && !signal)) return RCABEAM_ERROR_ARGUMENT;
  if (nv > kStaticMaxVoxels || ns > INT32_MAX || nc > INT32_MAX || na > INT32_MAX || nt > INT32_MAX ||
      nc * na > INT32_MAX || na > 4096)
    return RCABEAM_ERROR_ARGUMENT;
  void* scratch = static_scratch_address();
  if (!scratch) return RCABEAM_ERROR_CUDA;
  // The sort's scratch for the largest accepted call must fit the array (the
  // radix-sort temporaries depend on the CUB version): checked once, on the host.
  static const bool fits = order_bytes(kStaticMaxVoxels, nullptr) <= kStaticScratchBytes;
  if (!fits) return RCABEAM_ERROR_CUDA;
  if (cudaMemsetAsync(pd, 0, 2 * nv * sizeof(float), 0) != cudaSuccess) return RCABEAM_ERROR_CUDA;
  das::Args a{};
  a.rc = rc;
  a.cr = cr;
  a.scan = scan;
  a.xe = xe;
  a.ye = ye;
  a.angles = angles;
  a.starts = starts;
  a.pd = pd;
  a.signal = static_cast<float2*>(signal);
  a.ns = int(ns);
  a.nc = int(nc);
  a.na = int(na);
  a.nt = int(nt);
  a.nv = int(nv);
  a.c = double(c);
  a.fs = double(fs);
  a.fd = double(fd);
  a.fn = double(fn);
  a.err = device_error_ptr();
  if (method == 2) {
    dim3 grid(unsigned((nv + generic::kWarps - 1) / generic::kWarps),
              unsigned((nt + 32 * generic::kRegFrames - 1) / (32 * generic::kRegFrames)));
    generic::ensemble_nonlinear<2><<<grid, generic::kWarps * 32>>>(a);
    return launch_status();
  }
  // The sort rewrites keys, values and the bounding box (cleared inside) on every call.
  // Calls too small to need an order run in identity order; a failed sort is an error.
  a.order = voxel_order(scan, nv, scratch, kStaticScratchBytes);
  if (!a.order && order_bytes(nv, nullptr)) return RCABEAM_ERROR_CUDA;
  if (method == 3) return run_dmas_staged(a, (nv + das::kTileVoxels - 1) / das::kTileVoxels);
  const size_t ntiles = (nv + das::kTileVoxels - 1) / das::kTileVoxels;
  rcabeam_status st = method == 0   ? run_staged<false, das::kOpw>(a, ntiles)
                      : method == 5 ? run_staged<false, das::kApertures>(a, ntiles)
                                    : run_staged<false, das::kXdoppler>(a, ntiles);
  if (st != RCABEAM_SUCCESS) return st;
  if (method == 1) {
    das::finish_magnitude<<<unsigned((nv + 255) / 256), 256>>>(pd, nv);
    return launch_status();
  }
  return RCABEAM_SUCCESS;
}

}  // namespace rcb

using namespace rcb;

extern "C" {

const char* rcabeam_status_string(rcabeam_status status) {
  switch (status) {
    case RCABEAM_SUCCESS: return "success";
    case RCABEAM_ERROR_CUDA: return "cuda error";
    case RCABEAM_ERROR_ARGUMENT: return "invalid argument";
  }
  return "unknown error";
}

// ------------------------------------------------ clutter-filter extensions --
rcabeam_status rcabeam_clutter_scale_device(const void* iq, size_t n, int complex128, double* scale) {
  if (!iq || !scale || !n) return RCABEAM_ERROR_ARGUMENT;
  auto* out = reinterpret_cast<unsigned long long*>(scale);
  if (complex128)
    clutter::max_abs_kernel<double2><<<296, 256>>>(static_cast<const double2*>(iq), n, out);
  else if (reinterpret_cast<uintptr_t>(iq) % 16 == 0) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t want = (n / 2 + 4 * 256 - 1) / (4 * 256);  // four float4 per thread
    const unsigned blocks = unsigned(std::max<size_t>(1, std::min<size_t>(want, size_t(sms) * 8)));
    clutter::max_abs_c64<<<blocks, 256>>>(static_cast<const float2*>(iq), n, out);
  } else {
    clutter::max_abs_kernel<float2><<<296, 256>>>(static_cast<const float2*>(iq), n, out);
  }
  return launch_status();
}

// Tensor-core Gram (precision 2 = TF32, 3 = 3xBF16) of a complex64 Casorati
// matrix: the rows x 2T float32 view as a 2-D tensor with 32 x 16 SWIZZLE_128B
// boxes, one CTA per (unit, row slice).
static rcabeam_status gram_tc_launch(const void* iq, size_t rows, size_t nt, const double* scale, bool tf32,
                                     double* upper) {
  auto fn = encode_fn();
  if (!fn) return RCABEAM_ERROR_CUDA;
  gramtc::Params prm{};
  const int nb = int((2 * nt + gramtc::kBlock - 1) / gramtc::kBlock);
  prm.nunits = gramtc::plan_units(nb, prm.units, &prm.nload_max);
  if (!prm.nunits) return RCABEAM_ERROR_ARGUMENT;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  prm.slices = sms / prm.nunits > 0 ? sms / prm.nunits : 1;
  const size_t per = (rows + prm.slices - 1) / prm.slices;
  prm.slice_rows = (long long)((per + gramtc::kRows - 1) / gramtc::kRows * gramtc::kRows);
  prm.slices = int((rows + prm.slice_rows - 1) / prm.slice_rows);
  prm.rows = (long long)rows;
  prm.nt = int(nt);
  prm.scale = scale;
  prm.upper = upper;
  prm.err = device_error_ptr();
  CUtensorMap map;
  cuuint64_t dims[2] = {2 * nt, rows};
  cuuint64_t strides[1] = {2 * nt * 4};
  cuuint32_t box[2] = {32, cuuint32_t(gramtc::kRows)};
  cuuint32_t estr[2] = {1, 1};
  if (fn(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(iq), dims, strides, box, estr,
         CU_TENSOR_MAP_INTERLEAVE_NONE, tf32 ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return RCABEAM_ERROR_ARGUMENT;
  // The deepest rings that fit 227 KB (units stage at most three blocks: four
  // 3xBF16 staging and operand stages, eight TF32 stages); at least 120 KB
  // keeps one CTA (and one 512-column TMEM allocation) per SM.
  prm.ring = 2;
  while (prm.ring < gramtc::kMaxRing && gramtc::smem_bytes(prm.nload_max, prm.ring + 1) <= (size_t(227) << 10))
    ++prm.ring;
  const size_t smem = std::max(gramtc::smem_bytes(prm.nload_max, prm.ring), size_t(120) << 10);
  auto kern = tf32 ? gramtc::gram_tc<true> : gramtc::gram_tc<false>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  kern<<<unsigned(prm.nunits * prm.slices), gramtc::kThreads, smem>>>(map, prm);
  return launch_status();
}

rcabeam_status rcabeam_gram_accumulate_device(const void* iq, size_t rows, size_t nt, int complex128,
                                              const double* scale, int precision, double* upper) {
  if (!iq || !scale || !upper || !rows || !nt || nt > 65535) return RCABEAM_ERROR_ARGUMENT;
  if (precision < 0 || precision > 3) return RCABEAM_ERROR_ARGUMENT;
  if (precision >= 2) {
    // complex64 rows whose 8 nt-byte stride is a multiple of 16; T <= 1024; rows < 2^31.
    if (complex128 || nt % 2 || nt > 1024 || rows >= (size_t(1) << 31) ||
        reinterpret_cast<uintptr_t>(iq) % 16 != 0)
      return RCABEAM_ERROR_ARGUMENT;
    return gram_tc_launch(iq, rows, nt, scale, precision == 2, upper);
  }
  int nb = int((nt + clutter::kGramTile - 1) / clutter::kGramTile);
  unsigned tiles = unsigned(nb * (nb + 1) / 2);
  size_t want = (148 * 8 + tiles - 1) / tiles;
  size_t slices = (rows + clutter::kGramRows - 1) / clutter::kGramRows;
  if (slices > want) slices = want;
  if (slices > 65535) slices = 65535;
  dim3 grid(tiles, unsigned(slices));
  if (precision == 0) {
    if (complex128)
      clutter::gram_simt<double, double2><<<grid, clutter::kGramThreads>>>(static_cast<const double2*>(iq), rows,
                                                                          int(nt), scale, nb, upper);
    else
      clutter::gram_simt<double, float2><<<grid, clutter::kGramThreads>>>(static_cast<const float2*>(iq), rows,
                                                                         int(nt), scale, nb, upper);
  } else {
    if (complex128)
      clutter::gram_simt<float, double2><<<grid, clutter::kGramThreads>>>(static_cast<const double2*>(iq), rows,
                                                                         int(nt), scale, nb, upper);
    else
      clutter::gram_simt<float, float2><<<grid, clutter::kGramThreads>>>(static_cast<const float2*>(iq), rows,
                                                                        int(nt), scale, nb, upper);
  }
  return launch_status();
}

rcabeam_status rcabeam_gram_finish_device(const double* upper, double* gram, size_t nt, size_t total_rows) {
  if (!upper || !gram || !nt || !total_rows || nt > 65535) return RCABEAM_ERROR_ARGUMENT;
  dim3 grid(blocks_for(nt, 128), unsigned(nt));
  clutter::gram_finish<<<grid, 128>>>(upper, gram, int(nt), 1.0 / double(total_rows));
  return launch_status();
}

rcabeam_status rcabeam_heevd_workspace_bytes(size_t nt, size_t* bytes) {
  if (!bytes || !nt || nt > 65535) return RCABEAM_ERROR_ARGUMENT;
  cusolverDnHandle_t h = solver_handle();
  if (!h) return RCABEAM_ERROR_CUDA;
  int lwork = 0;
  if (cusolverDnZheevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, int(nt), nullptr, int(nt),
                                  nullptr, &lwork) != CUSOLVER_STATUS_SUCCESS)
    return RCABEAM_ERROR_CUDA;
  *bytes = size_t(lwork) * sizeof(cuDoubleComplex);
  return RCABEAM_SUCCESS;
}

rcabeam_status rcabeam_heevd_device(double* gram, double* eigenvalues, size_t nt, void* workspace,
                                    size_t workspace_bytes, int* info) {
  if (!gram || !eigenvalues || !workspace || !info || !nt || nt > 65535) return RCABEAM_ERROR_ARGUMENT;
  cusolverDnHandle_t h = solver_handle();
  if (!h) return RCABEAM_ERROR_CUDA;
  if (cusolverDnSetStream(h, 0) != CUSOLVER_STATUS_SUCCESS) return RCABEAM_ERROR_CUDA;
  int lwork = int(workspace_bytes / sizeof(cuDoubleComplex));
  if (cusolverDnZheevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, int(nt),
                       reinterpret_cast<cuDoubleComplex*>(gram), int(nt), eigenvalues,
                       static_cast<cuDoubleComplex*>(workspace), lwork, info) != CUSOLVER_STATUS_SUCCESS)
    return RCABEAM_ERROR_CUDA;
  return launch_status();
}

rcabeam_status rcabeam_project_device(const void* iq, void* out, double* power, size_t rows, size_t nt,
                                      int complex128, const double* vectors, size_t k, int mode, unsigned* flags) {
  if (!iq || !rows || !nt || nt > 512 || (k && !vectors) || mode < 0 || mode > 3 || ((mode & 2) && !out) ||
      (!power && !(mode & 2)))
    return RCABEAM_ERROR_ARGUMENT;
  if (complex128)
    project_dispatch<double2>(iq, out, power, rows, nt, vectors, k, mode, flags);
  else
    project_dispatch<float2>(iq, out, power, rows, nt, vectors, k, mode, flags);
  return launch_status();
}

rcabeam_status rcabeam_ritz_matrix_device(const void* iq, size_t rows, size_t nt, const double* vectors, size_t m,
                                         double* h) {
  if (!iq || !vectors || !h || !rows || !nt || nt > 512 || !m || m > size_t(clutter::kRitzMax) ||
      reinterpret_cast<uintptr_t>(iq) % 8 != 0)
    return RCABEAM_ERROR_ARGUMENT;
  if (cudaMemsetAsync(h, 0, m * m * 2 * sizeof(double), 0) != cudaSuccess) return RCABEAM_ERROR_CUDA;
  const size_t smem = size_t(clutter::kRitzMax) * clutter::ritz_stride(int(nt)) * 16 +
                      size_t(clutter::kRefineRows) * clutter::kRitzMax * 16 + size_t(clutter::kRefineRows) * nt * 8;
  if (cudaFuncSetAttribute(clutter::ritz_matrix, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) !=
      cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t blocks = std::min<size_t>(size_t(sms) * 3, (rows + clutter::kRefineRows - 1) / clutter::kRefineRows);
  clutter::ritz_matrix<<<unsigned(blocks), clutter::kRitzThreads, smem>>>(
      static_cast<const float2*>(iq), rows, int(nt), reinterpret_cast<const double2*>(vectors), int(m), h);
  return launch_status();
}

rcabeam_status rcabeam_ensemble_workspace_bytes(size_t nv, size_t nc, size_t na, size_t* bytes) {
  if (!bytes || !nv || !nc || !na) return RCABEAM_ERROR_ARGUMENT;
  size_t need = order_bytes(nv, nullptr);
  size_t documented = 2 * nv * (nc + na) * 16;
  *bytes = need ? (need < documented ? need : documented) : 256;
  return RCABEAM_SUCCESS;
}

rcabeam_status rcabeam_ensemble_static_device(const void* rc, const void* cr, const float* scan, const float* xe,
                                              const float* ye, const float* angles, const float* starts, float* pd,
                                              void* signal, size_t ns, size_t nc, size_t na, size_t nt, size_t nv,
                                              float c, float fs, float fd, float fn, int method) {
  return ensemble_static(rc, cr, scan, xe, ye, angles, starts, pd, signal, ns, nc, na, nt, nv, c, fs, fd, fn,
                         method);
}

rcabeam_status rcabeam_wait_selftest_device(unsigned long long limit_ns, int code, int* gave_up) {
  if (!gave_up || code <= 0 || limit_ns == 0 || limit_ns > kWaitLimitNs) return RCABEAM_ERROR_ARGUMENT;
  int* err = device_error_ptr();
  if (!err) return RCABEAM_ERROR_CUDA;
  wait_selftest<<<1, 128>>>(err, code, limit_ns, gave_up);
  return launch_status();
}

rcabeam_status rcabeam_device_error(int* code) {
  if (!code) return RCABEAM_ERROR_ARGUMENT;
  if (cudaDeviceSynchronize() != cudaSuccess) return RCABEAM_ERROR_CUDA;
  int zero = 0;
  if (cudaMemcpyFromSymbol(code, g_device_error, sizeof(int)) != cudaSuccess) return RCABEAM_ERROR_CUDA;
  if (cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int)) != cudaSuccess) return RCABEAM_ERROR_CUDA;
  return RCABEAM_SUCCESS;
}

rcabeam_status rcabeam_pack_ensemble_device(const void* source, void* target, size_t ns, size_t nc, size_t na,
                                            size_t nt) {
  if (!source || !target || !ns || !nc || !na || !nt || ns > SIZE_MAX / nc / na / nt) return RCABEAM_ERROR_ARGUMENT;
  return launch_pack<false>(source, target, nullptr, ns, nc, na, nt);
}

rcabeam_status rcabeam_pack_ensemble_fp16_device(const void* source, void* target, int* range_error, size_t ns,
                                                 size_t nc, size_t na, size_t nt) {
  if (!source || !target || !range_error || !ns || !nc || !na || !nt || ns > SIZE_MAX / nc / na / nt ||
      reinterpret_cast<uintptr_t>(source) % alignof(float2) != 0 ||
      reinterpret_cast<uintptr_t>(target) % alignof(__half2) != 0 ||
      reinterpret_cast<uintptr_t>(range_error) % alignof(int) != 0)
    return RCABEAM_ERROR_ARGUMENT;
  return launch_pack<true>(source, target, range_error, ns, nc, na, nt);
}

rcabeam_status rcabeam_ensemble_device(const void* rc, const void* cr, const float* scan, const float* xe,
                                       const float* ye, const float* angles, const float* starts, float* pd,
                                       void* signal, float* weights, void* workspace, void* geometry_workspace,
                                       size_t ns, size_t nc, size_t na, size_t nt, size_t nv, float c, float fs,
                                       float fd, float fn, int method, int k) {
  return ensemble_impl<false>(rc, cr, scan, xe, ye, angles, starts, pd, signal, weights, workspace,
                              geometry_workspace, ns, nc, na, nt, nv, c, fs, fd, fn, method, k);
}

rcabeam_status rcabeam_pack_ensemble_split_device(const void* source, void* hi, void* lo, int* range_error, size_t ns,
                                                  size_t nc, size_t na, size_t nt) {
  if (!source || !hi || !lo || !range_error || !ns || !nc || !na || !nt || ns > SIZE_MAX / nc / na / nt ||
      reinterpret_cast<uintptr_t>(source) % alignof(float2) != 0 || reinterpret_cast<uintptr_t>(hi) % 4 != 0 ||
      reinterpret_cast<uintptr_t>(lo) % 4 != 0 || reinterpret_cast<uintptr_t>(range_error) % alignof(int) != 0)
    return RCABEAM_ERROR_ARGUMENT;
  size_t rows = ns * nc * na;
  size_t blocks = (rows + kPackThreads / 32 - 1) / (kPackThreads / 32);
  if (blocks > 148ull * 64ull) blocks = 148ull * 64ull;
  pack_split_rows<<<unsigned(blocks), kPackThreads>>>(static_cast<const float2*>(source),
                                                      static_cast<__nv_bfloat162*>(hi),
                                                      static_cast<__nv_bfloat162*>(lo), range_error, ns, nc, na, nt);
  return launch_status();
}

rcabeam_status rcabeam_opw_tc_device(const void* rc_hi, const void* rc_lo, const void* cr_hi, const void* cr_lo,
                                     const float* scan, const float* xe, const float* ye, const float* angles,
                                     const float* starts, float* pd, void* signal, void* geometry_workspace,
                                     size_t ns, size_t nc, size_t na, size_t nt, size_t nv, float c, float fs,
                                     float fd, float fn, int precision) {
  if (!rc_hi || !cr_hi || !scan || !xe || !ye || !angles || !starts || !pd || !geometry_workspace || ns < 2 ||
      !nc || !na || !nt || !nv || c <= 0 || fs <= 0 || !std::isfinite(c) || !std::isfinite(fs) ||
      !std::isfinite(fd) || !std::isfinite(fn) || precision < 0 || precision > 3)
    return RCABEAM_ERROR_ARGUMENT;
  if (ns > INT32_MAX || nc * na > INT32_MAX || nt > INT32_MAX || nv > size_t(INT32_MAX) - tc::kVox || na > 4096)
    return RCABEAM_ERROR_ARGUMENT;
  const bool bf16x3 = precision & 1;
  const void* planes[4] = {rc_hi, cr_hi, rc_lo, cr_lo};
  if (!tc_eligible(planes, bf16x3 ? 4 : 2, nt)) return RCABEAM_ERROR_ARGUMENT;
  if (cudaMemsetAsync(pd, 0, 2 * nv * sizeof(float), 0) != cudaSuccess) return RCABEAM_ERROR_CUDA;
  tc::Args t{};
  t.x_hi[0] = rc_hi;
  t.x_hi[1] = cr_hi;
  t.x_lo[0] = rc_lo;
  t.x_lo[1] = cr_lo;
  t.scan = scan;
  t.xe = xe;
  t.ye = ye;
  t.angles = angles;
  t.starts = starts;
  t.order = voxel_order(scan, nv, geometry_workspace, 2 * nv * (nc + na) * 16);
  t.pd = pd;
  t.signal = static_cast<float2*>(signal);
  t.ns = int(ns);
  t.nc = int(nc);
  t.na = int(na);
  t.nt = int(nt);
  t.nv = int(nv);
  t.c = c;
  t.fs = fs;
  t.fd = fd;
  t.fn = fn;
  t.err = device_error_ptr();
  t.walk_fixed = (precision & 2) ? 1 : 0;
  return bf16x3 ? run_tc<true>(t) : run_tc<false>(t);
}

rcabeam_status rcabeam_opw_fp16_device(const void* rc, const void* cr, const float* scan, const float* xe,
                                       const float* ye, const float* angles, const float* starts, float* pd,
                                       void* signal, void* geometry_workspace, size_t ns, size_t nc, size_t na,
                                       size_t nt, size_t nv, float c, float fs, float fd, float fn) {
  if (reinterpret_cast<uintptr_t>(rc) % alignof(__half2) != 0 ||
      reinterpret_cast<uintptr_t>(cr) % alignof(__half2) != 0)
    return RCABEAM_ERROR_ARGUMENT;
  return ensemble_impl<true>(rc, cr, scan, xe, ye, angles, starts, pd, signal, nullptr, nullptr, geometry_workspace,
                             ns, nc, na, nt, nv, c, fs, fd, fn, 0, 2);
}

// ------------------------------------------------- single-frame API --
rcabeam_status rcabeam_opw_device(const void* iq, void* out, size_t n_voxels, size_t n_angles, size_t n_frames) {
  if (!iq || !out || !n_voxels || !n_angles || !n_frames) return RCABEAM_ERROR_ARGUMENT;
  generic::angles_opw<<<blocks_for(n_voxels * n_frames, 256), 256>>>(static_cast<const float2*>(iq),
                                                                      static_cast<float2*>(out), n_voxels, n_angles,
                                                                      n_frames);
  return launch_status();
}

static rcabeam_status angle_pd(const void* iq, float* out, size_t nv, size_t na, size_t nt, size_t rs, size_t rn,
                               size_t cs, size_t cn, int fmas) {
  if (!iq || !out || !nv || !na || !nt) return RCABEAM_ERROR_ARGUMENT;
  if (rs + rn > na || cs + cn > na) return RCABEAM_ERROR_ARGUMENT;
  generic::angles_pd<<<blocks_for(nv, 256), 256>>>(static_cast<const float2*>(iq), out, nv, na, nt, rs, rn, cs, cn,
                                                   fmas);
  return launch_status();
}

rcabeam_status rcabeam_xdoppler_pd_device(const void* iq, float* out, size_t n_voxels, size_t n_angles,
                                          size_t n_frames, size_t rc_start, size_t rc_count, size_t cr_start,
                                          size_t cr_count) {
  return angle_pd(iq, out, n_voxels, n_angles, n_frames, rc_start, rc_count, cr_start, cr_count, 0);
}

rcabeam_status rcabeam_rc_fmas_pd_device(const void* iq, float* out, size_t n_voxels, size_t n_angles,
                                         size_t n_frames, size_t rc_start, size_t rc_count, size_t cr_start,
                                         size_t cr_count) {
  return angle_pd(iq, out, n_voxels, n_angles, n_frames, rc_start, rc_count, cr_start, cr_count, 1);
}

rcabeam_status rcabeam_delay_rca_channels_device(const void* iq_ch, const float* scan_coords_m,
                                                 const float* elements_m, const float* angles_rad,
                                                 const float* t_start_s, void* out, size_t n_samples,
                                                 size_t n_channels, size_t n_angles, size_t n_voxels, int config,
                                                 float sound_speed_m_s, float sampling_freq_hz, float demod_freq_hz,
                                                 float f_number) {
  if (bad_frame_args(iq_ch, scan_coords_m, elements_m, angles_rad, t_start_s, out, n_samples, n_channels, n_angles,
                     n_voxels, config))
    return RCABEAM_ERROR_ARGUMENT;
  auto f = frame_args(iq_ch, nullptr, scan_coords_m, elements_m, elements_m, angles_rad, t_start_s, n_samples,
                      n_channels, n_angles, n_voxels, sound_speed_m_s, sampling_freq_hz, demod_freq_hz, f_number);
  generic::frame_angle_sums<<<blocks_for(n_voxels * n_angles, 128), 128>>>(f, config, static_cast<float2*>(out));
  return launch_status();
}

rcabeam_status rcabeam_delay_rca_channel_data_device(const void* iq_ch, const float* scan_coords_m,
                                                     const float* elements_m, const float* angles_rad,
                                                     const float* t_start_s, void* channel_sum, void* angle_sum,
                                                     float* n_active, size_t n_samples, size_t n_channels,
                                                     size_t n_angles, size_t n_voxels, int config,
                                                     float sound_speed_m_s, float sampling_freq_hz,
                                                     float demod_freq_hz, float f_number) {
  if (bad_frame_args(iq_ch, scan_coords_m, elements_m, angles_rad, t_start_s, angle_sum, n_samples, n_channels,
                     n_angles, n_voxels, config) ||
      !channel_sum || !n_active)
    return RCABEAM_ERROR_ARGUMENT;
  auto f = frame_args(iq_ch, nullptr, scan_coords_m, elements_m, elements_m, angles_rad, t_start_s, n_samples,
                      n_channels, n_angles, n_voxels, sound_speed_m_s, sampling_freq_hz, demod_freq_hz, f_number);
  generic::frame_angle_sums<<<blocks_for(n_voxels * n_angles, 128), 128>>>(f, config,
                                                                             static_cast<float2*>(angle_sum));
  generic::frame_channel_sums<<<blocks_for(n_voxels * n_channels, 128), 128>>>(
      f, config, static_cast<float2*>(channel_sum), n_active);
  return launch_status();
}

static rcabeam_status frame_pd(const void* iq_rc, const void* iq_cr, const float* scan, const float* xe,
                               const float* ye, const float* angles, const float* starts, int which, float* o_opw,
                               float* o_xd, float* o_fmas, float* o_dmas, size_t ns, size_t nc, size_t na, size_t nv,
                               float c, float fs, float fd, float fn) {
  float* first = o_opw ? o_opw : (o_xd ? o_xd : (o_fmas ? o_fmas : o_dmas));
  if (bad_frame_args(iq_rc, scan, xe, angles, starts, first, ns, nc, na, nv, 0) || !iq_cr || !ye)
    return RCABEAM_ERROR_ARGUMENT;
  auto f = frame_args(iq_rc, iq_cr, scan, xe, ye, angles, starts, ns, nc, na, nv, c, fs, fd, fn);
  generic::frame_reduce<<<blocks_for(nv, 128), 128>>>(f, which, o_opw, o_xd, o_fmas, o_dmas);
  return launch_status();
}

rcabeam_status rcabeam_opw_pd_from_channels_device(const void* iq_rc, const void* iq_cr, const float* scan_coords_m,
                                                   const float* x_elements_m, const float* y_elements_m,
                                                   const float* angles_rad, const float* t_start_s, float* out,
                                                   size_t n_samples, size_t n_channels, size_t n_angles,
                                                   size_t n_voxels, float sound_speed_m_s, float sampling_freq_hz,
                                                   float demod_freq_hz, float f_number) {
  if (!out) return RCABEAM_ERROR_ARGUMENT;
  return frame_pd(iq_rc, iq_cr, scan_coords_m, x_elements_m, y_elements_m, angles_rad, t_start_s,
                  generic::kFrameOpw, out, nullptr, nullptr, nullptr, n_samples, n_channels, n_angles, n_voxels,
                  sound_speed_m_s, sampling_freq_hz, demod_freq_hz, f_number);
}

rcabeam_status rcabeam_xdoppler_pd_from_channels_device(const void* iq_rc, const void* iq_cr,
                                                        const float* scan_coords_m, const float* x_elements_m,
                                                        const float* y_elements_m, const float* angles_rad,
                                                        const float* t_start_s, float* out, size_t n_samples,
                                                        size_t n_channels, size_t n_angles, size_t n_voxels,
                                                        float sound_speed_m_s, float sampling_freq_hz,
                                                        float demod_freq_hz, float f_number) {
  if (!out) return RCABEAM_ERROR_ARGUMENT;
  return frame_pd(iq_rc, iq_cr, scan_coords_m, x_elements_m, y_elements_m, angles_rad, t_start_s, generic::kFrameXd,
                  nullptr, out, nullptr, nullptr, n_samples, n_channels, n_angles, n_voxels, sound_speed_m_s,
                  sampling_freq_hz, demod_freq_hz, f_number);
}

rcabeam_status rcabeam_rc_fmas_pd_from_channels_device(const void* iq_rc, const void* iq_cr,
                                                       const float* scan_coords_m, const float* x_elements_m,
                                                       const float* y_elements_m, const float* angles_rad,
                                                       const float* t_start_s, float* out, size_t n_samples,
                                                       size_t n_channels, size_t n_angles, size_t n_voxels,
                                                       float sound_speed_m_s, float sampling_freq_hz,
                                                       float demod_freq_hz, float f_number) {
  if (!out) return RCABEAM_ERROR_ARGUMENT;
  return frame_pd(iq_rc, iq_cr, scan_coords_m, x_elements_m, y_elements_m, angles_rad, t_start_s,
                  generic::kFrameFmas, nullptr, nullptr, out, nullptr, n_samples, n_channels, n_angles, n_voxels,
                  sound_speed_m_s, sampling_freq_hz, demod_freq_hz, f_number);
}

rcabeam_status rcabeam_fast_pd_from_channels_device(const void* iq_rc, const void* iq_cr, const float* scan_coords_m,
                                                    const float* x_elements_m, const float* y_elements_m,
                                                    const float* angles_rad, const float* t_start_s, float* opw_out,
                                                    float* xdoppler_out, float* rc_fmas_out, size_t n_samples,
                                                    size_t n_channels, size_t n_angles, size_t n_voxels,
                                                    float sound_speed_m_s, float sampling_freq_hz,
                                                    float demod_freq_hz, float f_number) {
  if (!opw_out || !xdoppler_out || !rc_fmas_out) return RCABEAM_ERROR_ARGUMENT;
  return frame_pd(iq_rc, iq_cr, scan_coords_m, x_elements_m, y_elements_m, angles_rad, t_start_s,
                  generic::kFrameOpw | generic::kFrameXd | generic::kFrameFmas, opw_out, xdoppler_out, rc_fmas_out,
                  nullptr, n_samples, n_channels, n_angles, n_voxels, sound_speed_m_s, sampling_freq_hz,
                  demod_freq_hz, f_number);
}

rcabeam_status rcabeam_dmas_ccf_acf_from_channels_device(const void* iq_rc, const void* iq_cr,
                                                         const float* scan_coords_m, const float* x_elements_m,
                                                         const float* y_elements_m, const float* angles_rad,
                                                         const float* t_start_s, float* out, size_t n_samples,
                                                         size_t n_channels, size_t n_angles, size_t n_voxels,
                                                         float sound_speed_m_s, float sampling_freq_hz,
                                                         float demod_freq_hz, float f_number) {
  if (!out) return RCABEAM_ERROR_ARGUMENT;
  return frame_pd(iq_rc, iq_cr, scan_coords_m, x_elements_m, y_elements_m, angles_rad, t_start_s,
                  generic::kFrameDmas, nullptr, nullptr, nullptr, out, n_samples, n_channels, n_angles, n_voxels,
                  sound_speed_m_s, sampling_freq_hz, demod_freq_hz, f_number);
}

}  // extern "C"

// ------------------------------------------------- differentiable OPW --
static bool adjoint_geometry(adj::Geometry* g, const float* scan, const unsigned* voxels, size_t nvl,
                             const float* xe, const float* ye, const float* angles, const float* starts,
                             const double* offsets, double c, float fs, float fd, float fn, size_t ns, size_t nc,
                             size_t na, size_t nt, size_t frame0, size_t frames) {
  if (!scan || !xe || !ye || !angles || !starts || !offsets || !nvl || ns < 2 || !nc || !na || !nt || !frames ||
      frames > size_t(adj::kChunk) || frame0 + frames > nt || !(c > 0) || !(fs > 0) || !std::isfinite(c) ||
      !std::isfinite(fs) || !std::isfinite(fd) || !std::isfinite(fn) || nvl > INT32_MAX || ns > INT32_MAX ||
      nc > 65535 || na > 65535 || nt > INT32_MAX)
    return false;
  g->scan = scan;
  g->voxels = voxels;
  g->xe = xe;
  g->ye = ye;
  g->angles = angles;
  g->starts = starts;
  g->offsets = offsets;
  g->c = c;
  g->fs = fs;
  g->fd = fd;
  g->fn = fn;
  g->nvl = int(nvl);
  g->ns = int(ns);
  g->nc = int(nc);
  g->na = int(na);
  g->nt = int(nt);
  g->f0 = int(frame0);
  g->frames = int(frames);
  return true;
}

rcabeam_status rcabeam_opw_offsets_forward_device(const void* rc, const void* cr, const float* scan,
                                                  const unsigned* voxels, size_t nvl, const float* xe,
                                                  const float* ye, const float* angles, const float* starts,
                                                  const double* offsets, double c, float fs, float fd, float fn,
                                                  size_t ns, size_t nc, size_t na, size_t nt, size_t frame0,
                                                  size_t frames, void* iq, double* power, int complex128) {
  adj::Geometry g;
  if (!rc || !cr || (!iq && !power) ||
      !adjoint_geometry(&g, scan, voxels, nvl, xe, ye, angles, starts, offsets, c, fs, fd, fn, ns, nc, na, nt, frame0,
                        frames))
    return RCABEAM_ERROR_ARGUMENT;
  const unsigned blocks = unsigned((nvl + 127) / 128);
  if (complex128)
    adj::forward<double><<<blocks, 128>>>(g, static_cast<const double2*>(rc), static_cast<const double2*>(cr),
                                          static_cast<double2*>(iq), power);
  else
    adj::forward<float><<<blocks, 128>>>(g, static_cast<const float2*>(rc), static_cast<const float2*>(cr),
                                         static_cast<float2*>(iq), power);
  return launch_status();
}

rcabeam_status rcabeam_opw_offsets_power_device(const void* rc, const void* cr, const float* scan, const float* xe,
                                                const float* ye, const float* angles, const float* starts,
                                                const double* offsets, double c, float fs, float fd, float fn,
                                                size_t ns, size_t nc, size_t na, size_t nt, size_t nv, float* pd,
                                                void* workspace, size_t workspace_bytes) {
  if (!rc || !cr || !scan || !xe || !ye || !angles || !starts || !offsets || !pd || !workspace || ns < 2 || !nc ||
      !na || !nt || !nv || !(c > 0) || !(fs > 0) || !std::isfinite(c) || !std::isfinite(fs) || !std::isfinite(fd) ||
      !std::isfinite(fn) || ns > INT32_MAX || nc > INT32_MAX || na > 4096 || nt > INT32_MAX || nv > INT32_MAX ||
      nc * na > INT32_MAX)
    return RCABEAM_ERROR_ARGUMENT;
  if (cudaMemsetAsync(pd, 0, 2 * nv * sizeof(float), 0) != cudaSuccess) return RCABEAM_ERROR_CUDA;
  das::Args a{};
  a.rc = rc;
  a.cr = cr;
  a.scan = scan;
  a.xe = xe;
  a.ye = ye;
  a.angles = angles;
  a.starts = starts;
  a.pd = pd;
  a.ns = int(ns);
  a.nc = int(nc);
  a.na = int(na);
  a.nt = int(nt);
  a.nv = int(nv);
  a.c = c;
  a.fs = double(fs);
  a.fd = double(fd);
  a.fn = double(fn);
  a.err = device_error_ptr();
  a.offsets = offsets;
  a.order = voxel_order(scan, nv, workspace, workspace_bytes);
  return run_staged<false, das::kOpw>(a, (nv + das::kTileVoxels - 1) / das::kTileVoxels);
}

rcabeam_status rcabeam_opw_offsets_adjoint_device(const void* rc, const void* cr, const float* scan,
                                                  const unsigned* voxels, size_t nvl, const float* xe,
                                                  const float* ye, const float* angles, const float* starts,
                                                  const double* offsets, double c, float fs, float fd, float fn,
                                                  size_t ns, size_t nc, size_t na, size_t nt, size_t frame0,
                                                  size_t frames, const void* grad_iq, void* grad_rc, void* grad_cr,
                                                  double* grad_offsets, double* grad_c, int complex128) {
  adj::Geometry g;
  if (!rc || !cr || !grad_iq || !grad_rc || !grad_cr || !grad_offsets || !grad_c ||
      !adjoint_geometry(&g, scan, voxels, nvl, xe, ye, angles, starts, offsets, c, fs, fd, fn, ns, nc, na, nt, frame0,
                        frames))
    return RCABEAM_ERROR_ARGUMENT;
  const size_t threads = nvl * 2 * nc;
  const unsigned blocks = unsigned((threads + 127) / 128);
  if (complex128)
    adj::adjoint<double><<<blocks, 128>>>(g, static_cast<const double2*>(rc), static_cast<const double2*>(cr),
                                          static_cast<const double2*>(grad_iq), static_cast<double2*>(grad_rc),
                                          static_cast<double2*>(grad_cr), grad_offsets, grad_c);
  else
    adj::adjoint<float><<<blocks, 128>>>(g, static_cast<const float2*>(rc), static_cast<const float2*>(cr),
                                         static_cast<const float2*>(grad_iq), static_cast<float2*>(grad_rc),
                                         static_cast<float2*>(grad_cr), grad_offsets, grad_c);
  return launch_status();
}

// ---------------------------------------------------------- batch queue --
namespace {
struct BatchLayout {
  size_t ens, maps, next, done, tile_done, total;
};

bool batch_plan(size_t n, const rcabeam_batch_ensemble* list, std::vector<batch::Ensemble>* out, BatchLayout* L,
                long long* total_items) {
  if (!n || !list || n > (1u << 20)) return false;
  long long items = 0, tiles_xd = 0;
  if (out) out->resize(n);
  for (size_t i = 0; i < n; ++i) {
    const rcabeam_batch_ensemble& d = list[i];
    if (!d.rc || !d.cr || !d.scan || !d.xe || !d.ye || !d.angles || !d.starts || !d.pd || d.ns < 2 || !d.nc ||
        !d.na || !d.nt || !d.nv || d.na > size_t(batch::kMaxAngles) || d.nv > INT32_MAX || d.ns > INT32_MAX ||
        d.nc > INT32_MAX || d.nt > INT32_MAX || !(d.c > 0) || !(d.fs > 0) || !std::isfinite(d.c) ||
        !std::isfinite(d.fs) || !std::isfinite(d.fd) || !std::isfinite(d.fn))
      return false;
    if (d.method != 0 && d.method != 1 && d.method != 3) return false;
    const int fpc = d.frames_per_chunk ? d.frames_per_chunk : 64;
    if (fpc != 16 && fpc != 32 && fpc != 64) return false;
    batch::Ensemble e{};
    e.method = d.method;
    e.lpv = fpc / 2;
    if (d.method == 3) {
      e.lpv = batch::kDmasLpv;
      e.tiles = int((d.nv + das::kTileVoxels - 1) / das::kTileVoxels);
      e.chunks = int((d.nt + 2 * batch::kDmasLpv - 1) / (2 * batch::kDmasLpv));
    } else {
      // Whole F-frame chunks, then one tail chunk of the next power of two >= 4 frames.
      e.tiles = int((d.nv + das::kTileVoxels - 1) / das::kTileVoxels);
      e.main_chunks = int(d.nt / fpc);
      const unsigned tail = unsigned(d.nt % fpc);
      e.lpv_tail = tail ? int(std::max(pow2_at_least(tail), 4u) / 2) : 0;
      e.chunks = e.main_chunks + (tail ? 1 : 0);
    }
    e.tma = (d.nt * 8) % 16 == 0 && reinterpret_cast<uintptr_t>(d.rc) % 16 == 0 &&
            reinterpret_cast<uintptr_t>(d.cr) % 16 == 0 && encode_fn() != nullptr;
    e.first_item = items;
    e.tile_base = tiles_xd;
    items += (long long)e.tiles * e.chunks;
    if (d.method == 1) tiles_xd += e.tiles;
    das::Args& a = e.args;
    a.rc = d.rc;
    a.cr = d.cr;
    a.scan = d.scan;
    a.xe = d.xe;
    a.ye = d.ye;
    a.angles = d.angles;
    a.starts = d.starts;
    a.order = d.order;
    a.pd = d.pd;
    a.signal = nullptr;
    a.ns = int(d.ns);
    a.nc = int(d.nc);
    a.na = int(d.na);
    a.nt = int(d.nt);
    a.nv = int(d.nv);
    a.c = d.c;
    a.fs = d.fs;
    a.fd = d.fd;
    a.fn = d.fn;
    a.frame_base = 0;
    a.err = device_error_ptr();
    if (out) (*out)[i] = e;
  }
  L->ens = 0;
  L->maps = align256(n * sizeof(batch::Ensemble));
  L->next = L->maps + align256(4 * n * sizeof(CUtensorMap));
  L->done = L->next + 256;
  L->tile_done = L->done + align256(n * 4);
  L->total = L->tile_done + align256(size_t(tiles_xd > 0 ? tiles_xd : 1) * 4);
  *total_items = items;
  return true;
}

batch::Queue batch_queue(void* table, size_t n, const BatchLayout& L, long long total, unsigned long long* times) {
  unsigned char* t = static_cast<unsigned char*>(table);
  batch::Queue q{};
  q.ens = reinterpret_cast<const batch::Ensemble*>(t + L.ens);
  q.maps = reinterpret_cast<const CUtensorMap*>(t + L.maps);
  q.n = int(n);
  q.total_items = total;
  q.next = reinterpret_cast<unsigned long long*>(t + L.next);
  q.done = reinterpret_cast<unsigned*>(t + L.done);
  q.tile_done = reinterpret_cast<unsigned*>(t + L.tile_done);
  q.times = times;
  q.err = device_error_ptr();
  return q;
}
}  // namespace

extern "C" {

rcabeam_status rcabeam_batch_table_bytes(size_t n, const rcabeam_batch_ensemble* list, size_t* bytes) {
  BatchLayout L;
  long long total = 0;
  if (!bytes || !batch_plan(n, list, nullptr, &L, &total)) return RCABEAM_ERROR_ARGUMENT;
  *bytes = L.total;
  return RCABEAM_SUCCESS;
}

rcabeam_status rcabeam_batch_prepare(size_t n, const rcabeam_batch_ensemble* list, void* table,
                                     size_t table_bytes) {
  BatchLayout L;
  long long total = 0;
  std::vector<batch::Ensemble> ens;
  if (!table || reinterpret_cast<uintptr_t>(table) % 256 != 0 || !batch_plan(n, list, &ens, &L, &total) ||
      table_bytes < L.total)
    return RCABEAM_ERROR_ARGUMENT;
  std::vector<CUtensorMap> maps(4 * n);
  for (size_t i = 0; i < n; ++i) {
    batch::Ensemble& e = ens[i];
    if (!e.tma) continue;
    const size_t slabs = size_t(e.args.nc) * e.args.na, nt = size_t(e.args.nt), ns = size_t(e.args.ns);
    for (int part = 0; part < 2; ++part) {
      const int frames = 2 * (part ? e.lpv_tail : e.lpv);
      if (!frames) continue;
      if (!make_slab_map(&maps[4 * i + 2 * part], e.args.rc, 8, nt, ns, slabs, frames, das::kRows) ||
          !make_slab_map(&maps[4 * i + 2 * part + 1], e.args.cr, 8, nt, ns, slabs, frames, das::kRows))
        return RCABEAM_ERROR_ARGUMENT;  // the run's kernel variant follows the plan's tma flags
    }
  }
  unsigned char* t = static_cast<unsigned char*>(table);
  if (cudaMemcpy(t + L.ens, ens.data(), n * sizeof(batch::Ensemble), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t + L.maps, maps.data(), 4 * n * sizeof(CUtensorMap), cudaMemcpyHostToDevice) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  return RCABEAM_SUCCESS;
}

rcabeam_status rcabeam_batch_run_device(size_t n, const rcabeam_batch_ensemble* list, void* table,
                                        size_t table_bytes, unsigned long long* times, int ctas_per_sm,
                                        void* stream) {
  BatchLayout L;
  long long total = 0;
  if (!table || !times || ctas_per_sm < 0 || ctas_per_sm > 3 || !batch_plan(n, list, nullptr, &L, &total) ||
      table_bytes < L.total)
    return RCABEAM_ERROR_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* t = static_cast<unsigned char*>(table);
  // Counters, completion times (start slot = all ones for the atomicMin) and every power map.
  if (cudaMemsetAsync(t + L.next, 0, L.total - L.next, st) != cudaSuccess ||
      cudaMemsetAsync(times, 0xff, 8, st) != cudaSuccess || cudaMemsetAsync(times + 1, 0, 8 * n, st) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  for (size_t i = 0; i < n; ++i)
    if (cudaMemsetAsync(list[i].pd, 0, 2 * list[i].nv * sizeof(float), st) != cudaSuccess) return RCABEAM_ERROR_CUDA;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  std::vector<batch::Ensemble> ens;
  batch_plan(n, list, &ens, &L, &total);
  if (ctas_per_sm == 0) {
    // Grid mode: each ensemble through the single-ensemble kernels on the
    // stream (for ensembles that fill the GPU alone, where those kernels run
    // faster than the persistent loop), a completion stamp after each.
    batch::stamp<<<1, 1, 0, st>>>(times, 1);
    for (size_t i = 0; i < n; ++i) {
      const das::Args& a = ens[i].args;
      const size_t ntiles = (size_t(a.nv) + das::kTileVoxels - 1) / das::kTileVoxels;
      rcabeam_status r = RCABEAM_SUCCESS;
      if (list[i].method == 3) {
        r = run_dmas_staged(a, ntiles, st);
      } else if (list[i].method == 1) {
        r = run_staged<false, das::kXdoppler>(a, ntiles, st);
        if (r == RCABEAM_SUCCESS) das::finish_magnitude<<<unsigned((a.nv + 255) / 256), 256, 0, st>>>(a.pd, a.nv);
      } else {
        r = run_staged<false, das::kOpw>(a, ntiles, st);
      }
      if (r != RCABEAM_SUCCESS) return r;
      batch::stamp<<<1, 1, 0, st>>>(times + 1 + i, 0);
    }
    return cudaGetLastError() == cudaSuccess ? RCABEAM_SUCCESS : RCABEAM_ERROR_CUDA;
  }
  // A queue of one method whose ensembles all stage the same way (TMA or plain
  // loads) at two or three CTAs per SM runs the kernel compiled for that
  // method and staging alone; anything else runs the general kernel.
  int kind = list[0].method, tma = ens[0].tma;
  for (size_t i = 1; i < n; ++i) {
    if (list[i].method != kind) kind = -1;
    if (ens[i].tma != tma) tma = -1;
  }
  using Kernel = void (*)(const batch::Queue);
  static const Kernel general[3] = {batch::run<1, -1, -1>, batch::run<2, -1, -1>, batch::run<3, -1, -1>};
  static const Kernel special[3][2][2] = {  // [kind][tma][ctas_per_sm - 2]
      {{batch::run<2, 0, 0>, batch::run<3, 0, 0>}, {batch::run<2, 0, 1>, batch::run<3, 0, 1>}},
      {{batch::run<2, 1, 0>, batch::run<3, 1, 0>}, {batch::run<2, 1, 1>, batch::run<3, 1, 1>}},
      {{batch::run<2, 3, 0>, batch::run<3, 3, 0>}, {batch::run<2, 3, 1>, batch::run<3, 3, 1>}},
  };
  const bool specific = kind >= 0 && tma >= 0 && ctas_per_sm >= 2;
  const Kernel kern = specific ? special[kind == 3 ? 2 : kind][tma][ctas_per_sm - 2] : general[ctas_per_sm - 1];
  const size_t smem = specific && kind == 3 ? batch::Smem<batch::smem_lpv<3>()>::kBytes : batch::Smem<32>::kBytes;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  const long long want = (long long)sms * ctas_per_sm;
  const unsigned grid = unsigned(total < want ? total : want);
  kern<<<grid, das::kThreads, smem, st>>>(batch_queue(table, n, L, total, times));
  return cudaGetLastError() == cudaSuccess ? RCABEAM_SUCCESS : RCABEAM_ERROR_CUDA;
}

rcabeam_status rcabeam_simulate_scene_device(const float* scatterers, size_t n, const float* elements,
                                             const float* angles, const float* starts, void* out, size_t ns,
                                             size_t nc, size_t na, size_t nt, int config, double prf, double c,
                                             double fs, double fd, double sigma_t, double half_width) {
  if (!scatterers || !elements || !angles || !starts || !out || !n || ns < 2 || !nc || !na || !nt ||
      (config != 0 && config != 1) || !(prf > 0) || !(c > 0) || !(fs > 0) || !std::isfinite(fd) ||
      !(sigma_t > 0) || !(half_width > 0) || ns > 16384 || nc * na > 65535 || nt > INT32_MAX ||
      n > SIZE_MAX / scene::kFields)
    return RCABEAM_ERROR_ARGUMENT;
  // Frame chunk: the (samples x chunk) complex64 slab stays within 96 KB (two CTAs per SM).
  size_t chunk = (96 * 1024) / (ns * sizeof(float2));
  if (chunk < 1) chunk = 1;
  if (chunk > nt) chunk = nt;
  const size_t smem = ns * chunk * sizeof(float2);
  if (cudaFuncSetAttribute(scene::simulate, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return RCABEAM_ERROR_CUDA;
  scene::Args a{};
  a.scatterers = scatterers;
  a.n = n;
  a.elements = elements;
  a.angles = angles;
  a.starts = starts;
  a.out = static_cast<float2*>(out);
  a.ns = int(ns);
  a.nc = int(nc);
  a.na = int(na);
  a.nt = int(nt);
  a.chunk = int(chunk);
  a.config = config;
  a.prf = prf;
  a.c = c;
  a.fs = fs;
  a.fd = fd;
  a.sigma = sigma_t;
  a.half_width = half_width;
  const dim3 grid(unsigned(nc * na), unsigned((nt + chunk - 1) / chunk));
  scene::simulate<<<grid, scene::kThreads, smem>>>(a);
  return launch_status();
}

rcabeam_status rcabeam_voxel_order_workspace_bytes(size_t nv, size_t* bytes) {
  if (!bytes) return RCABEAM_ERROR_ARGUMENT;
  *bytes = order_bytes(nv, nullptr);
  return *bytes ? RCABEAM_SUCCESS : RCABEAM_ERROR_ARGUMENT;
}

rcabeam_status rcabeam_voxel_order_device(const float* scan, size_t nv, unsigned* order, void* workspace,
                                          size_t workspace_bytes) {
  if (!scan || !order || !nv || !workspace) return RCABEAM_ERROR_ARGUMENT;
  const unsigned* sorted = voxel_order(scan, nv, workspace, workspace_bytes);
  if (!sorted) return RCABEAM_ERROR_ARGUMENT;
  return cudaMemcpyAsync(order, sorted, nv * sizeof(unsigned), cudaMemcpyDeviceToDevice, 0) == cudaSuccess
             ? RCABEAM_SUCCESS
             : RCABEAM_ERROR_CUDA;
}

}  // extern "C"
