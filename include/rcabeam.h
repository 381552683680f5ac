/* rcabeam C ABI -- B200 (sm_100a) implementation.
 *
 * Every declaration in the first part keeps the exact name, argument order,
 * types and status semantics of the reference interface include/rcabeam.h of
 * sdiebolt/rcabeam; the comment above each one cites the reference line it
 * replaces.  Declarations under "Extensions" have no reference C counterpart:
 * they expose the clutter filter (a CuPy module in the reference) and the
 * device error word of the bounded-wait kernels.
 *
 * All pointers are device pointers unless stated otherwise.  Work is launched
 * on the legacy default CUDA stream, as in the reference (rcabeam.h:200),
 * except rcabeam_batch_run_device, which takes a stream so that it can be
 * captured into a CUDA graph; calls return once the work is enqueued.  Nothing
 * here allocates device memory except the clutter-filter extensions, which say
 * so (the library's fixed scratch arrays are static device memory).
 */
#pragma once

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* reference rcabeam.h:9-13 */
typedef enum rcabeam_status {
    RCABEAM_SUCCESS = 0,
    RCABEAM_ERROR_CUDA = 1,
    RCABEAM_ERROR_ARGUMENT = 2,
} rcabeam_status;

/* reference rcabeam.h:15 */
const char* rcabeam_status_string(rcabeam_status status);

/* ---- Per-frame entry points (reference rcabeam.h:17-182; core.cu). ------
 * Single-frame channel layout is (samples, channels, angles) complex64;
 * per-angle IQ is (voxels, angles, frames).  config 0 = RC, 1 = CR.
 * f_number <= 0 keeps the full receive aperture. */

/* reference rcabeam.h:17-23: out[v, t] = sum over angles of iq[v, a, t]. */
rcabeam_status rcabeam_opw_device(const void* iq, void* out, size_t n_voxels, size_t n_angles, size_t n_frames);

/* reference rcabeam.h:25-35: |mean_t (sum RC angles)(sum CR angles)^*|. */
rcabeam_status rcabeam_xdoppler_pd_device(const void* iq, float* out, size_t n_voxels, size_t n_angles,
                                          size_t n_frames, size_t rc_start, size_t rc_count, size_t cr_start,
                                          size_t cr_count);

/* reference rcabeam.h:37-47: mean_t |(sum sqrt RC)(sum sqrt CR)|^2. */
rcabeam_status rcabeam_rc_fmas_pd_device(const void* iq, float* out, size_t n_voxels, size_t n_angles,
                                         size_t n_frames, size_t rc_start, size_t rc_count, size_t cr_start,
                                         size_t cr_count);

/* reference rcabeam.h:49-65: per-angle DAS volumes out[v, a] of one frame. */
rcabeam_status rcabeam_delay_rca_channels_device(const void* iq_ch, const float* scan_coords_m,
                                                 const float* elements_m, const float* angles_rad,
                                                 const float* t_start_s, void* out, size_t n_samples,
                                                 size_t n_channels, size_t n_angles, size_t n_voxels, int config,
                                                 float sound_speed_m_s, float sampling_freq_hz, float demod_freq_hz,
                                                 float f_number);

/* reference rcabeam.h:67-85: channel sums [v, c], angle sums [v, a], active counts [v]. */
rcabeam_status rcabeam_delay_rca_channel_data_device(const void* iq_ch, const float* scan_coords_m,
                                                     const float* elements_m, const float* angles_rad,
                                                     const float* t_start_s, void* channel_sum, void* angle_sum,
                                                     float* n_active, size_t n_samples, size_t n_channels,
                                                     size_t n_angles, size_t n_voxels, int config,
                                                     float sound_speed_m_s, float sampling_freq_hz,
                                                     float demod_freq_hz, float f_number);

/* reference rcabeam.h:87-104: |sum RC + CR|^2 of one frame. */
rcabeam_status rcabeam_opw_pd_from_channels_device(const void* iq_rc, const void* iq_cr, const float* scan_coords_m,
                                                   const float* x_elements_m, const float* y_elements_m,
                                                   const float* angles_rad, const float* t_start_s, float* out,
                                                   size_t n_samples, size_t n_channels, size_t n_angles,
                                                   size_t n_voxels, float sound_speed_m_s, float sampling_freq_hz,
                                                   float demod_freq_hz, float f_number);

/* reference rcabeam.h:106-123: |RC conj(CR)| of one frame. */
rcabeam_status rcabeam_xdoppler_pd_from_channels_device(const void* iq_rc, const void* iq_cr,
                                                        const float* scan_coords_m, const float* x_elements_m,
                                                        const float* y_elements_m, const float* angles_rad,
                                                        const float* t_start_s, float* out, size_t n_samples,
                                                        size_t n_channels, size_t n_angles, size_t n_voxels,
                                                        float sound_speed_m_s, float sampling_freq_hz,
                                                        float demod_freq_hz, float f_number);

/* reference rcabeam.h:125-142: |(sum_a sqrt RC_a)(sum_a sqrt CR_a)|^2 of one frame. */
rcabeam_status rcabeam_rc_fmas_pd_from_channels_device(const void* iq_rc, const void* iq_cr,
                                                       const float* scan_coords_m, const float* x_elements_m,
                                                       const float* y_elements_m, const float* angles_rad,
                                                       const float* t_start_s, float* out, size_t n_samples,
                                                       size_t n_channels, size_t n_angles, size_t n_voxels,
                                                       float sound_speed_m_s, float sampling_freq_hz,
                                                       float demod_freq_hz, float f_number);

/* reference rcabeam.h:144-163: OPW, XDoppler and RC-FMAS of one frame in one pass. */
rcabeam_status rcabeam_fast_pd_from_channels_device(const void* iq_rc, const void* iq_cr, const float* scan_coords_m,
                                                    const float* x_elements_m, const float* y_elements_m,
                                                    const float* angles_rad, const float* t_start_s, float* opw_out,
                                                    float* xdoppler_out, float* rc_fmas_out, size_t n_samples,
                                                    size_t n_channels, size_t n_angles, size_t n_voxels,
                                                    float sound_speed_m_s, float sampling_freq_hz,
                                                    float demod_freq_hz, float f_number);

/* reference rcabeam.h:165-182: DMAS * CCF * ACF of one frame. */
rcabeam_status rcabeam_dmas_ccf_acf_from_channels_device(const void* iq_rc, const void* iq_cr,
                                                         const float* scan_coords_m, const float* x_elements_m,
                                                         const float* y_elements_m, const float* angles_rad,
                                                         const float* t_start_s, float* out, size_t n_samples,
                                                         size_t n_channels, size_t n_angles, size_t n_voxels,
                                                         float sound_speed_m_s, float sampling_freq_hz,
                                                         float demod_freq_hz, float f_number);

/* ---- Frame-batched ensemble path (the OPW hot path). ------------------- */

/* reference rcabeam.h:184-185: (samples, channels, angles, frames) complex64 ->
 * (channels, angles, samples, frames) complex64.  Source and target must not alias. */
rcabeam_status rcabeam_pack_ensemble_device(const void* source, void* target, size_t ns, size_t nc, size_t na,
                                            size_t nt);

/* reference rcabeam.h:187-207.  rc, cr: packed (channels, angles, samples, frames)
 * complex64.  method: 0 OPW, 1 XDoppler, 2 RC-FMAS, 3 DMAS-CCF-ACF, 4 St-SW,
 * 5 separate RC/CR IQ.  pd: 2*nv floats, the result is in the even entries.
 * signal: optional complex64 (nv, nt) output ((nv, 2, nt) for method 5).
 * weights/workspace: St-SW only: weights[nv] receives the raw St-SW weights
 * (normalize by their full-volume maximum before multiplying pd), workspace is
 * complex64 [nv * k * k * nt] correlation-series scratch, 2 <= k <= 4, na >= k,
 * signal must be null.  geometry_workspace: caller-owned scratch of
 * 2*nv*(nc+na) float4; this implementation computes delays on the fly and uses
 * the scratch only for its voxel traversal order.  Delays and phases are formed
 * in float64; interpolation and accumulation are float32. */
rcabeam_status rcabeam_ensemble_device(const void* rc, const void* cr, const float* scan, const float* xe,
                                       const float* ye, const float* angles, const float* starts, float* pd,
                                       void* signal, float* weights, void* workspace, void* geometry_workspace,
                                       size_t ns, size_t nc, size_t na, size_t nt, size_t nv, float c, float fs,
                                       float fd, float fn, int method, int k);

/* reference rcabeam.h:209-220: pack to complex FP16 (two IEEE halves, RN).
 * range_error (one device int, zeroed by the caller) is set to 1 when a
 * component is non-finite or beyond +/-65504. */
rcabeam_status rcabeam_pack_ensemble_fp16_device(const void* source, void* target, int* range_error, size_t ns,
                                                 size_t nc, size_t na, size_t nt);

/* reference rcabeam.h:222-235: OPW from FP16-packed RC/CR; float32 geometry
 * interpolation and accumulation, complex64 signal. */
rcabeam_status rcabeam_opw_fp16_device(const void* rc, const void* cr, const float* scan, const float* xe,
                                       const float* ye, const float* angles, const float* starts, float* pd,
                                       void* signal, void* geometry_workspace, size_t ns, size_t nc, size_t na,
                                       size_t nt, size_t nv, float c, float fs, float fd, float fn);

/* ---- Extensions (no counterpart in the reference C interface). ---------- */

/* Packs complex64 (samples, channels, angles, frames) into two planes of
 * (channels, angles, samples, frames) BF16 (re, im) pairs: hi = bf16(x) and
 * lo = bf16(x - hi), the split operand of the three-product tensor-core OPW.
 * range_error (one device int, zeroed by the caller) is set to 1 when a
 * component is not finite.  Source must be 8-byte aligned; hi, lo 4-byte. */
rcabeam_status rcabeam_pack_ensemble_split_device(const void* source, void* hi, void* lo, int* range_error, size_t ns,
                                                  size_t nc, size_t na, size_t nt);

/* OPW IQ and power on tcgen05 tensor cores (interpolation as a banded GEMM
 * over 64-voxel tiles).  precision bit 0 clear: rc_hi / cr_hi are FP16-packed
 * channels (rcabeam_pack_ensemble_fp16_device), rc_lo / cr_lo unused; bit 0
 * set: BF16 hi / lo planes from rcabeam_pack_ensemble_split_device.  Bit 1 set:
 * every tile starts its channel walk at the same slot (clear: each tile starts
 * where the other SMs are, which keeps their sample windows in L2 together but
 * makes the order of the float32 sums depend on timing); the interleaving of
 * the builder warps still varies, so repeated calls agree to about 1e-7 of the
 * IQ instead of being bit-identical; the unaligned walk costs about 10 % more
 * time (more of its windows miss L2).  Coefficients are
 * split into hi + lo halves; accumulation is float32.  pd, signal and
 * geometry_workspace are as for rcabeam_ensemble_device (method 0).  Requires
 * nt % 4 == 0 and 16-byte aligned planes (RCABEAM_ERROR_ARGUMENT otherwise).
 * rcabeam_opw_fp16_device uses this kernel whenever its inputs qualify. */
rcabeam_status rcabeam_opw_tc_device(const void* rc_hi, const void* rc_lo, const void* cr_hi, const void* cr_lo,
                                     const float* scan, const float* xe, const float* ye, const float* angles,
                                     const float* starts, float* pd, void* signal, void* geometry_workspace,
                                     size_t ns, size_t nc, size_t na, size_t nt, size_t nv, float c, float fs,
                                     float fd, float fn, int precision);

/* Clutter filter (reference src/rcabeam/gpu_clutter.py, a CuPy module there).
 * IQ is a row-major (rows, nt) Casorati matrix, complex64 (complex128 = 0) or
 * complex128 (complex128 = 1).  Gram and basis matrices are complex128. */

/* *scale (device double, zeroed by the caller) = max(|re|, |im|) over n values
 * (gpu_clutter.py:141); infinite for an infinite component and NaN for a NaN
 * one, so a finite scale certifies finite input (gpu_clutter.py:36-37). */
rcabeam_status rcabeam_clutter_scale_device(const void* iq, size_t n, int complex128, double* scale);

/* Adds the upper-triangle tiles of (X / s)^H (X / s), s = *scale (1 if zero),
 * into upper (device, row-major nt x nt complex128, zeroed by the caller).
 * precision: 0 float64 CUDA cores, 1 float32 CUDA cores, 2 TF32 tensor cores,
 * 3 3xBF16 tensor cores.  Precisions 2 and 3 (tcgen05, float32 accumulation
 * flushed to float64 every 2048 rows) need complex64 rows (complex128 = 0),
 * an even nt <= 1024, rows < 2^31 and a 16-byte aligned iq; they scale X by
 * the power of two that bounds s before rounding, so the sum stays in range.
 * Call once per array to estimate one shared basis (gpu_clutter.py:144-160). */
rcabeam_status rcabeam_gram_accumulate_device(const void* iq, size_t rows, size_t nt, int complex128,
                                              const double* scale, int precision, double* upper);

/* gram (device, column-major nt x nt complex128) = (G + G^H) / (2 total_rows)
 * from the accumulated upper tiles (gpu_clutter.py:160-161). */
rcabeam_status rcabeam_gram_finish_device(const double* upper, double* gram, size_t nt, size_t total_rows);

/* Float64 Hermitian eigendecomposition of gram (cuSOLVER zheevd): ascending
 * eigenvalues; gram is overwritten by the column eigenvectors.  workspace holds
 * rcabeam_heevd_workspace_bytes bytes; *info (device int) is the solver status. */
rcabeam_status rcabeam_heevd_workspace_bytes(size_t nt, size_t* bytes);
rcabeam_status rcabeam_heevd_device(double* gram, double* eigenvalues, size_t nt, void* workspace,
                                    size_t workspace_bytes, int* info);

/* Per row x: coordinates y = x V on k column-major (nt x k) complex128 vectors.
 * mode bit 0: residual x - y V^H (else the retained part y V^H); bit 1: write
 * it to out (input dtype).  power (device double[rows], optional when writing)
 * receives |residual|^2 / nt, or sum |y|^2 / nt without bit 0 (gpu_clutter.py:196-273).
 * nt <= 512.  flags (device unsigned, optional, cleared by the caller) is ORed
 * with 1 when an input component is not finite and with 2 when a power is not
 * finite, the two checks gpu_clutter.py:25-40 and :271-272 make, in the same pass. */
rcabeam_status rcabeam_project_device(const void* iq, void* out, double* power, size_t rows, size_t nt,
                                      int complex128, const double* vectors, size_t k, int mode,
                                      unsigned* flags);

/* Float64 Rayleigh-Ritz matrix on complex64 rows X (extension): h (device,
 * m x m complex128, column-major; cleared inside) = (X V)^H (X V) for the m <= 16
 * vectors V (m x nt row-major complex128, vector c in row c, nt <= 512), i.e.
 * V^H (X^H X) V without forming the Gram.  Its eigenvectors rotate V onto the
 * float64 Gram's eigenvectors within span(V). */
rcabeam_status rcabeam_ritz_matrix_device(const void* iq, size_t rows, size_t nt, const double* vectors, size_t m,
                                         double* h);

/* Bytes of geometry_workspace that rcabeam_ensemble_device / rcabeam_opw_fp16_device
 * actually use for nv voxels (at most the documented 2*nv*(nc+na) float4).  A
 * buffer of this size may be passed instead of the documented one. */
rcabeam_status rcabeam_ensemble_workspace_bytes(size_t nv, size_t nc, size_t na, size_t* bytes);

/* Same computation as rcabeam_ensemble_device (methods 0, 1, 2, 3 and 5), for
 * callers that cannot allocate device memory -- acquisition loops whose memory
 * budget is fixed up front, plugins whose host owns the device allocator: it
 * takes no geometry workspace and keeps its scratch in a fixed 8 MiB array
 * inside the library, so the call itself never allocates.  No counterpart in
 * the reference interface.
 * Limits: nv <= 262144 voxels per call (RCABEAM_ERROR_ARGUMENT beyond, and for
 * method 4).  All calls on a device share the scratch: calls that overlap on
 * the GPU (other streams or threads) race.  The first call on each device
 * looks up the scratch address; make that first call before any stream
 * capture.  Launches use the legacy default stream. */
rcabeam_status rcabeam_ensemble_static_device(const void* rc, const void* cr, const float* scan, const float* xe,
                                              const float* ye, const float* angles, const float* starts, float* pd,
                                              void* signal, size_t ns, size_t nc, size_t na, size_t nt, size_t nv,
                                              float c, float fs, float fd, float fn, int method);

/* Differentiable OPW (extension; no counterpart in the reference interface).
 * The OPW model of rcabeam_ensemble_device (method 0) with a per-receive-
 * element delay offset offsets[A * nc + c] (seconds; A = 0 RC, 1 CR) added to
 * every delay and a float64 sound speed c.  rc, cr: channels in the USER
 * layout (ns, nc, na, nt), complex64 (complex128 = 0) or complex128.  voxels:
 * nvl indices into scan (null: the first nvl voxels).  One call covers frames
 * [frame0, frame0 + frames), frames <= 8.
 * Forward: iq (nvl x frames, the channels' complex type) and/or power (nvl
 * float64) += sum_t |IQ|^2 / nt. */
rcabeam_status rcabeam_opw_offsets_forward_device(const void* rc, const void* cr, const float* scan,
                                                  const unsigned* voxels, size_t nvl, const float* xe,
                                                  const float* ye, const float* angles, const float* starts,
                                                  const double* offsets, double c, float fs, float fd, float fn,
                                                  size_t ns, size_t nc, size_t na, size_t nt, size_t frame0,
                                                  size_t frames, void* iq, double* power, int complex128);

/* Power of the same model over nv voxels and every frame, from PACKED complex64
 * channels (rcabeam_pack_ensemble_device) on the TMA-staged float32 DAS: pd
 * (2 * nv floats, result in the even entries).  workspace: at least
 * rcabeam_ensemble_workspace_bytes(nv, nc, na) bytes (traversal order). */
rcabeam_status rcabeam_opw_offsets_power_device(const void* rc, const void* cr, const float* scan, const float* xe,
                                                const float* ye, const float* angles, const float* starts,
                                                const double* offsets, double c, float fs, float fd, float fn,
                                                size_t ns, size_t nc, size_t na, size_t nt, size_t nv, float* pd,
                                                void* workspace, size_t workspace_bytes);

/* Adjoint of rcabeam_opw_offsets_forward_device for the upstream gradient grad_iq (nvl x frames,
 * dL/dRe + j dL/dIm): adds to grad_rc / grad_cr (user layout, channels' type;
 * atomics), grad_offsets (2 * nc float64) and *grad_c (float64). */
rcabeam_status rcabeam_opw_offsets_adjoint_device(const void* rc, const void* cr, const float* scan,
                                                  const unsigned* voxels, size_t nvl, const float* xe,
                                                  const float* ye, const float* angles, const float* starts,
                                                  const double* offsets, double c, float fs, float fd, float fn,
                                                  size_t ns, size_t nc, size_t na, size_t nt, size_t frame0,
                                                  size_t frames, const void* grad_iq, void* grad_rc, void* grad_cr,
                                                  double* grad_offsets, double* grad_c, int complex128);

/* Batch queue (extension; no counterpart in the reference interface): a queue
 * of uneven ensembles reconstructed by one persistent kernel.  Each entry
 * describes one ensemble with packed (c, a, s, t) complex64 channels and its
 * own grid (scan, optional traversal order from rcabeam_voxel_order_device),
 * geometry, power output (2 * nv floats, result in the even entries) and
 * method: 0 OPW, 1 XDoppler, 3 DMAS-CCF-ACF.  frames_per_chunk (16, 32, 64;
 * 0 = 64) is the staged methods' frame chunk, chosen by an autotuner. */
typedef struct rcabeam_batch_ensemble {
  const void* rc;
  const void* cr;
  const float* scan;
  const unsigned* order;
  const float* xe;
  const float* ye;
  const float* angles;
  const float* starts;
  float* pd;
  size_t ns, nc, na, nt, nv;
  float c, fs, fd, fn;
  int method;
  int frames_per_chunk;
} rcabeam_batch_ensemble;

/* Device table bytes of a queue of n ensembles (angles <= 64 per ensemble). */
rcabeam_status rcabeam_batch_table_bytes(size_t n, const rcabeam_batch_ensemble* list, size_t* bytes);

/* Writes the queue's device table (256-byte aligned; synchronous copies): call
 * once per queue, before any stream capture of rcabeam_batch_run_device. */
rcabeam_status rcabeam_batch_prepare(size_t n, const rcabeam_batch_ensemble* list, void* table,
                                     size_t table_bytes);

/* Enqueues on `stream` (a cudaStream_t; capturable into a CUDA graph): clears
 * the counters and every pd, then runs the persistent kernel with ctas_per_sm
 * (1-3) CTAs per SM (a queue of one method runs that method's own kernel), or
 * with ctas_per_sm = 0 launches every ensemble through the single-ensemble
 * kernels in queue order.  times (device, n + 1 uint64): start, then each
 * ensemble's completion, in global-timer nanoseconds. */
rcabeam_status rcabeam_batch_run_device(size_t n, const rcabeam_batch_ensemble* list, void* table,
                                        size_t table_bytes, unsigned long long* times, int ctas_per_sm,
                                        void* stream);

/* Scene synthesis (extension; test and benchmark input, no counterpart in the
 * reference C interface).  Writes out = channel IQ (ns, nc, na, nt) complex64
 * of one aperture (config 0 = RC receiving on x elements, 1 = CR on y) for n
 * moving point scatterers, the Gaussian-pulse model of the reference's
 * simulate_point (src/rcabeam/sim.py:131-189):
 *   sum_k amp_k exp(-((t - tau)/sigma_t)^2) exp(-j 2 pi fd tau),
 * t = starts[a] + i / fs, evaluated where |t - tau| <= half_width.
 * scatterers: n x 11 floats (ox, oz, oy, dx, dz, dy, s0, speed, period,
 * amp_re, amp_im); at frame f (time f / prf) a scatterer sits at
 * o + d * s with s = s0 + speed * f / prf, wrapped into [0, period) when
 * period > 0.  Every element of out is written. */
rcabeam_status rcabeam_simulate_scene_device(const float* scatterers, size_t n, const float* elements,
                                             const float* angles, const float* starts, void* out, size_t ns,
                                             size_t nc, size_t na, size_t nt, int config, double prf, double c,
                                             double fs, double fd, double sigma_t, double half_width);

/* Workspace bytes of rcabeam_voxel_order_device for nv voxels (128 <= nv < 2^31). */
rcabeam_status rcabeam_voxel_order_workspace_bytes(size_t nv, size_t* bytes);

/* Spatially compact traversal order (Morton codes of the voxel positions,
 * radix-sorted) of nv voxels into order (nv unsigned), on the default stream. */
rcabeam_status rcabeam_voxel_order_device(const float* scan, size_t nv, unsigned* order, void* workspace,
                                          size_t workspace_bytes);

/* Failure-path self-test of the bounded waits (extension; no counterpart in the
 * reference): one CTA of four warps waits, limit_ns at most (<= 2 s), on an
 * mbarrier that nothing arrives on, with the same wait routine as the
 * staging pipelines.  Each wait gives up, sets the device error word to `code`
 * (> 0; read it with rcabeam_device_error) and returns; *gave_up (device int,
 * zeroed by the caller) counts the waits that gave up.  The context stays usable. */
rcabeam_status rcabeam_wait_selftest_device(unsigned long long limit_ns, int code, int* gave_up);

/* Reads and clears the device error word set by a kernel whose bounded wait
 * gave up (0 = no error).  Synchronizes the device. */
rcabeam_status rcabeam_device_error(int* code);

#ifdef __cplusplus
}
#endif
