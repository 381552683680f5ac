#!/usr/bin/env python
"""Benchmark of the OPW path on B200: full-size filtered OPW power Doppler.

Workload (one "step" = one ensemble): 128 + 128 element RCA, 0.11 mm pitch,
fs 20 MHz, f_demod 15 MHz, c 1540 m/s; complex64 IQ of 512 samples x 128
channels x 11 angles (-10..10 deg) x 200 frames per aperture; a 128 x 256 x 128
(x, z, y) grid over +-7 mm laterally and 4-12 mm in depth; full receive
aperture.  A step packs both apertures, beamforms OPW IQ with power, forms the
temporal Gram matrix, eigendecomposes it and reduces the clutter-filtered
power Doppler (rank_start = 3).

Input: the seeded flow scene rendered on the GPU by the forward-model kernel
(20,000 tissue speckle scatterers moving rigidly at 1 mm/s, 0 dB; 5,000 blood
scatterers at -40 dB flowing at 10-30 mm/s through a 1 mm-radius tube; complex
noise at -50 dB; PRF 500 Hz).

Metric: OPW samples/s, one sample = voxel x receive channel x angle x frame
over both apertures (2.362e12 per step), plus filtered-PD ms per ensemble.
Accuracy: every form's filtered power against the plain form on the whole
grid, and IQ / filtered power on a spread 2048-voxel sample against the
float64 C oracle (the filtered power of the oracle IQ uses the float64 basis of
the plain form's complex128 Gram).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU (torchrun): one independent ensemble per rank (weak scaling, no
data-path collective); rank 0 prints the JSON line with the max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NS, NC, NA, NT = 512, 128, 11, 200
GRID_SHAPE = (128, 256, 128)
PITCH = 0.11e-3
FS, FD, C = 20e6, 15e6, 1540.0
T_START = 4e-6
RANK_START = 3
# DRAM bytes (read + write) of one full-size bf16x3 tensor-core DAS launch, from
# an ncu capture of that launch (dram__bytes_read.sum + dram__bytes_write.sum).
DAS_DRAM_BYTES_PER_LAUNCH = 277_508_977_152 + 41_535_534_848
DAS_DRAM_SOURCE = ("ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum "
                   "--clock-control none -k regex:opw_tc -c 1 on the full-size flow-scene step (a 1-pass metric "
                   "set): 277.5 GB read + 41.5 GB written in one 797.6 ms launch; the writes are the 512-step "
                   "segment flushes into the complex64 IQ, the reads plane windows that missed L2")
# DAS unit model: FP32-equivalent operations per interpolated sample -- the
# lerp's two differences, two lerp FFMA and four FFMA of the complex rotate-
# accumulate -- against 128 FP32 lanes per SM per clock.
OPS_PER_UNIT = 8
SAMPLE_VOXELS = 2048


SUBGRID = None  # (nx, nz, ny) central block of the full grid, same spacing (profiling)


def workload():
    """Elements, angles and (x, z, y) grid of the workload (GRID_SHAPE may be reduced for profiling)."""
    el = (np.arange(NC) - (NC - 1) / 2) * PITCH
    angles = np.deg2rad(np.linspace(-10, 10, NA))
    half = (NC - 1) / 2 * PITCH
    grid = (np.linspace(-half, half, GRID_SHAPE[0]), np.linspace(4e-3, 12e-3, GRID_SHAPE[1]),
            np.linspace(-half, half, GRID_SHAPE[2]))
    if SUBGRID:
        grid = tuple(axis[(len(axis) - n) // 2:(len(axis) - n) // 2 + n] for axis, n in zip(grid, SUBGRID))
    return el, angles, grid


def units_per_step() -> int:
    return int(np.prod(SUBGRID or GRID_SHAPE)) * 2 * NC * NA * NT


CONFIG = {
    "workload": "filtered OPW PD: RCA 128+128 el 0.11 mm, IQ 512x128x11x200 c64 per aperture, grid 128x256x128, "
                "fs 20 MHz, f_demod 15 MHz, full aperture, SVD clutter filter rank_start=3",
    "samples": NS, "channels": NC, "angles": NA, "frames": NT, "grid": list(GRID_SHAPE),
    "l2": "inputs (2.3 GB packed channels, 6.7 GB IQ) are larger than L2; no flush",
}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.path.open("w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        rows = [r.split(", ") for r in self.path.read_text().splitlines() if r.count(",") >= 8]
        self.path.unlink(missing_ok=True)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": reasons}


def peaks() -> dict:
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except OSError:
        # The profiling recipe's fallback: copy 6.65 TB/s, cuBLAS bf16 1.59 PFLOP/s burst,
        # about 1.4 PFLOP/s sustained under the power cap (an earlier measurement on this pool).
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "fallback": True}


# ----------------------------------------------------------------- B200 arm --
FORMS = {
    # name: (packed IQ storage, Gram precision)
    "chosen": ("bf16x2", "bf16x3"),
    "plain": ("float32", "complex128"),
    "fp16_storage": ("float16", "complex128"),
}


def _time_form(plan, rc, cr, steps: int, warmup: int, world: int, clocks=None):
    """Device time of `steps` pipeline runs (max over ranks), after `warmup` runs."""
    import torch

    for _ in range(warmup):
        plan.run(rc, cr)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    das = []
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        torch.cuda.synchronize()
        start.record()
        for _ in range(steps):
            plan.run(rc, cr)
            das.append(plan.last_das_event_ms)
        stop.record()
        torch.cuda.synchronize()
    plan.check()
    elapsed = start.elapsed_time(stop) / 1e3
    if world > 1:
        t = torch.tensor([elapsed], device=rc.device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        elapsed = float(t.item())
    das_s = statistics.median(plan.collect_das_ms(e) for e in das) / 1e3
    return elapsed, das_s, plan.stage_ms()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def _scene(dev, seed: int):
    """The flow scene at the workload's shapes (on the workload's grid, or its profiling block)."""
    from rcabeam_b200 import scenes

    scene = scenes.flow_scene(channels=NC, pitch=PITCH, samples=NS, angles=NA, frames=NT, grid_shape=GRID_SHAPE,
                              t_start=T_START, seed=seed, device=dev)
    scene.grid = workload()[2]
    return scene


def _sample_ids(nv: int) -> np.ndarray:
    return np.unique(np.linspace(0, nv - 1, min(SAMPLE_VOXELS, nv)).round().astype(np.int64))


def _scene_accuracy(scene, sample_ids, iq_sample: dict, powers: dict, basis_plain: np.ndarray, rank_start: int):
    """IQ and filtered power of each form at the sample voxels against the float64 C oracle."""
    from oracle import c_das
    from rcabeam_b200.sim import scan_coords

    f32 = lambda v: np.asarray(v, dtype=np.float32).astype(np.float64)  # noqa: E731
    scan = scan_coords(scene.grid)[sample_ids].astype(np.float64)
    geom = scene.geom
    t0 = time.perf_counter()
    want = c_das.opw_iq(scene.rc.cpu().numpy(), scene.cr.cpu().numpy(), scan, f32(geom.x_el), f32(geom.y_el),
                        f32(scene.angles), f32([scene.t_start] * len(scene.angles)), float(np.float32(geom.c)),
                        float(np.float32(geom.fs)), float(np.float32(geom.f_demod)), None)
    oracle_s = time.perf_counter() - t0
    nt = want.shape[1]
    kept = basis_plain[:, rank_start:]
    want_pd = np.sum(np.abs(want @ kept) ** 2, axis=1) / nt
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    out = {"sample_voxels": int(len(sample_ids)), "oracle_seconds": round(oracle_s, 1)}
    for name, iq in iq_sample.items():
        out[f"{name}_iq_rel_l2_vs_f64"] = rel(iq, want)
        out[f"{name}_filtered_pd_rel_l2_vs_f64"] = rel(powers[name].cpu().numpy()[sample_ids], want_pd)
    return out


def run_b200(args, rank: int, world: int) -> dict | None:
    import torch

    from rcabeam_b200 import _lib, pipeline

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    scene = _scene(dev, seed=1234 + rank)
    rc, cr, angles, grid, geom = scene.rc, scene.cr, scene.angles, scene.grid, scene.geom
    torch.cuda.synchronize()
    units = units_per_step()
    sample_ids = _sample_ids(int(np.prod(SUBGRID or GRID_SHAPE)))
    results, powers, iq_sample = {}, {}, {}
    basis_plain = None
    clock = None
    for name in ("chosen", "plain", "fp16_storage"):
        if name != "chosen" and args.only_chosen:
            continue
        storage, precision = FORMS[name]
        plan = pipeline.FilteredOpw((NS, NC, NA, NT), angles, T_START, grid, geom, rank_start=RANK_START,
                                    precision=precision, iq_storage=storage)
        steps = args.steps if name == "chosen" else max(1, min(args.steps, 5))
        warm = args.warmup if name == "chosen" else min(args.warmup, 2)
        sampler = ClockSampler(dev.index) if name == "chosen" else None
        elapsed, das_s, stages = _time_form(plan, rc, cr, steps, warm, world, sampler)
        if sampler is not None:
            clock = sampler.summary()
        powers[name] = plan.power.clone()
        iq_sample[name] = plan.iq[torch.from_numpy(sample_ids).to(dev)].cpu().numpy()
        if name == "plain":
            nt = NT
            vt = torch.view_as_complex(plan.gram.matrix.view(nt, nt, 2)).cpu().numpy()  # rows: ascending eigvecs
            basis_plain = vt[::-1].T.copy()  # columns in descending order
        results[name] = {"ms_per_ensemble": round(elapsed / steps * 1e3, 3), "steps": steps,
                         "gsamples_per_s": round(units * world * steps / elapsed / 1e9, 3),
                         "das_ms": round(das_s * 1e3, 3), "stages_ms": stages, "iq_storage": storage,
                         "gram_precision": precision}
        if name == "chosen":
            # End to end through the public pipeline for a stream of ensembles: every step
            # uploads its channels from pinned host memory (overlapping the previous step's
            # reconstruction once that step has packed its channels) and reads its filtered
            # power back.
            host_rc, host_cr = rc.cpu().pin_memory(), cr.cpu().pin_memory()
            plan.run_host_sequence([(host_rc, host_cr)])
            e_steps = max(1, args.steps)
            outs = [torch.empty(plan.nv, dtype=torch.float64, pin_memory=True) for _ in range(e_steps)]
            torch.cuda.synchronize()
            e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e_start.record()
            plan.run_host_sequence([(host_rc, host_cr)] * e_steps, outs)
            e_stop.record()
            torch.cuda.synchronize()
            out = outs[-1]
            plan.check()
            e2e_s = e_start.elapsed_time(e_stop) / 1e3 / e_steps
            e2e = {"value": round(units / e2e_s / 1e9, 3), "unit": "Gsamples/s",
                   "ms_per_ensemble": round(e2e_s * 1e3, 3),
                   "h2d_bytes_per_step": int(host_rc.numel() * 8 * 2),
                   "d2h_bytes_per_step": int(out.numel() * out.element_size()), "steps": e_steps,
                   "mode": "FilteredOpw.run_host_sequence: per step pinned H2D of both apertures (side stream, "
                           "overlapping the previous step once it has packed) + reconstruction + D2H of the "
                           "filtered power"}
            launches = plan.launches_per_step()
            del host_rc, host_cr
        del plan
        torch.cuda.empty_cache()
    assert _lib.device_error() == 0
    accuracy = {}
    if "plain" in powers:
        ref = powers["plain"]
        for name in ("chosen", "fp16_storage"):
            accuracy[f"{name}_vs_plain_filtered_pd_rel_l2"] = float(
                torch.linalg.vector_norm(powers[name] - ref) / torch.linalg.vector_norm(ref))
        if rank == 0 and not args.no_accuracy:
            accuracy.update(_scene_accuracy(scene, sample_ids, iq_sample, powers, basis_plain, RANK_START))
    if rank != 0:
        return None
    ch = results["chosen"]
    pk = peaks()
    das_s = ch["das_ms"] / 1e3
    props = torch.cuda.get_device_properties(dev)
    sms = props.multi_processor_count
    mhz = (clock or {}).get("sm_mhz") or (clock or {}).get("sm_max_mhz") or 1965.0
    units_per_s = units / das_s
    fp32_peak = sms * 128 * mhz * 1e6  # FP32 lanes x clock (operations/s)
    # Tensor work issued by the dominant kernel: per (128-voxel tile, frame pass, aperture,
    # channel, angle) step, two 64-voxel groups x 3 products of one M=128 x N=2*frames x K=16
    # MMA (sub-window splits excluded).
    tiles = (int(np.prod(SUBGRID or GRID_SHAPE)) + 127) // 128
    passes = (NT + 127) // 128
    full = 128 if NT > 128 else (NT + 7) // 8 * 8
    pass_frames = [full] * (passes - 1) + [(NT - full * (passes - 1) + 7) // 8 * 8]
    mma_flops = tiles * 2 * NC * NA * 2 * 3 * 2 * 128 * sum(2 * f for f in pass_frames) * 16
    # Compulsory HBM bytes of one DAS launch: hi+lo packed planes read, IQ + power written.
    nvox = int(np.prod(SUBGRID or GRID_SHAPE))
    das_bytes = 2 * NS * NC * NA * NT * 8 + nvox * NT * 8 + nvox * 8
    tensor_peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops", 1590.0))
    peak_source = "fallback" if pk.get("fallback") else "measured"
    line = {
        "metric": "OPW Gsamples/s (vox*ch*ang*frm), filtered PD", "value": ch["gsamples_per_s"],
        "unit": "Gsamples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ch["ms_per_ensemble"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 math on bf16x2-split c64 IQ (tcgen05 3-product DAS), 3xBF16 tcgen05 Gram with f64 flushes, "
                 "f64 eig/projection",
        "data": "synthetic: seeded flow scene (tissue 0 dB at 1 mm/s, blood -40 dB at 10-30 mm/s in a 1 mm tube, "
                "noise -50 dB) rendered by the forward-model kernel at the full-size shapes",
        "config": {**CONFIG, "scene": scene.info["scene"], "scene_seed": scene.info["seed"]},
        "filtered_pd_ms_per_ensemble": {"chosen": ch["ms_per_ensemble"],
                                         **({"plain": results["plain"]["ms_per_ensemble"]} if "plain" in results else {})},
        "forms": results, "accuracy": accuracy, "e2e": e2e,
        "roofline": {
            "bound": "tensor", "kernel": "opw_tc<bf16x3> (DAS on tcgen05)",
            "achieved": round(OPS_PER_UNIT * units_per_s / 1e12, 2), "peak": round(fp32_peak / 1e12, 2),
            "unit": "TFLOP/s", "frac": round(OPS_PER_UNIT * units_per_s / fp32_peak, 4),
            "units_per_s": round(units_per_s, -6), "das_ms": ch["das_ms"],
            "model": f"FP32-issue-equivalent ceiling: {OPS_PER_UNIT} FP32 operations per interpolated sample "
                     f"(2 lerp differences, 2 lerp FFMA, 4 FFMA complex rotate-accumulate) x units/s, against "
                     f"{sms} SMs x 128 FP32 lanes x the median SM clock under load ({mhz:g} MHz); "
                     "frac = units/s / (SMs x 16 x clock)",
            "smem_gather_model": "16 B of shared-memory gathers per unit (2 float32 complex taps) at 128 B/clk/SM "
                                 "bounds a per-sample gather kernel (the SIMT float32 path); the tensor-core kernel "
                                 "stages each 16-row window once per 128-voxel tile and reads it through the MMA, "
                                 "so it does not bound this kernel",
            "issued_mma_tflops": round(mma_flops / das_s / 1e12, 1),
            "issued_mma_frac_of_bf16": round(mma_flops / das_s / 1e12 / tensor_peak, 4),
            "bf16_peak_tflops": tensor_peak, "peak_source": peak_source,
            # The capture is of the full-size launch: a reduced profiling workload has none.
            "traffic": None if "REDUCED" in CONFIG["workload"] else DAS_DRAM_BYTES_PER_LAUNCH,
            "traffic_source": ("not captured for a reduced workload" if "REDUCED" in CONFIG["workload"]
                               else DAS_DRAM_SOURCE),
            "compulsory_hbm_bytes": das_bytes,
            "note": f"compulsory HBM bytes {das_bytes / 1e9:.2f} GB per launch -> {das_bytes / das_s / 1e9:.1f} GB/s: "
                    "the DAS cannot be HBM-bound on algorithmic bytes"},
        "clocks": clock,
        "gpu_launches": launches * args.steps,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, voxels_per_core=args.cpu_voxels)
    return line


# --------------------------------------------------- batching form (queue) --
def run_batching(args) -> dict:
    """48 uneven ensembles (depth, frames, angles, method drawn from a seed) through the
    persistent queue kernel under a CUDA graph, next to sequential plain launches."""
    import torch

    from rcabeam_b200 import _lib, batching
    from rcabeam_b200.sim import RCAGeometry

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(args.seed)
    n = args.ensembles
    methods = ["opw"] * (n // 2) + ["xdoppler"] * (n // 4) + ["dmas"] * (n - n // 2 - n // 4)
    methods = [methods[i] for i in rng.permutation(n)]
    ns, nc = 512, 128
    el = (np.arange(nc) - (nc - 1) / 2) * PITCH
    half = (nc - 1) / 2 * PITCH
    geom = RCAGeometry(el, el, c=C, fs=FS, f_demod=FD, fnumber=None)
    dz = 8e-3 / 255
    gen = torch.Generator(device=dev).manual_seed(args.seed)
    ens, shapes = [], []
    for i in range(n):
        depth = int(rng.choice([128, 192, 256, 384]))
        nt = int(rng.choice([50, 100, 200, 400]))
        na = int(rng.choice([5, 7, 11]))
        chans = [torch.randn((ns * nc * na * nt,), dtype=torch.complex64, generator=gen, device=dev)
                 for _ in range(2)]
        lat = args.lateral
        grid = (np.linspace(-half, half, 128)[(128 - lat) // 2:(128 + lat) // 2], 4e-3 + dz * np.arange(depth),
                np.linspace(-half, half, 128)[(128 - lat) // 2:(128 + lat) // 2])
        e = batching.Ensemble(chans[0], chans[1], (ns, nc, na, nt), grid, geom,
                              np.deg2rad(np.linspace(-10, 10, na)), T_START, methods[i])
        e.build(dev)
        ens.append(e)
        shapes.append({"method": methods[i], "depth": depth, "frames": nt, "angles": na})
    torch.cuda.synchronize()
    tune_start = time.perf_counter()
    choice = batching.autotune(ens, sample_tiles=148 * 2, repeats=1)
    tune_s = time.perf_counter() - tune_start
    queue = batching.BatchQueue(ens, ctas_per_sm=choice["ctas_per_sm"])
    queue.capture()
    for _ in range(max(0, args.warmup - 1)):
        queue.run()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(1, args.steps)
    with ClockSampler(0) as sampler:
        start.record()
        for _ in range(steps):
            queue.run()
        stop.record()
        torch.cuda.synchronize()
    clocks = sampler.summary()
    assert _lib.device_error() == 0
    queue_ms = start.elapsed_time(stop) / steps
    done = queue.completion_ms()
    batch_pd = [e.power().clone() for e in ens]
    seq_done = batching.sequential(ens)
    worst = max(float(torch.linalg.vector_norm(b - e.power()) / torch.linalg.vector_norm(e.power()))
                for b, e in zip(batch_pd, ens))
    units = sum(e.units() for e in ens)
    durations = np.diff(np.concatenate(([0.0], seq_done)))
    by_method = {m: round(float(sum(d for d, e in zip(durations, ens) if e.method == m)), 1)
                 for m in ("opw", "xdoppler", "dmas")}
    return {
        "sequential_ms_by_method": by_method,
        "form": "batching", "metric": "ensembles/s, 48-ensemble uneven queue (OPW / XDoppler / DMAS-CCF-ACF)",
        "value": round(n / (queue_ms / 1e3), 4), "unit": "ensembles/s", "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_queue": round(queue_ms, 1),
        "latency_ms": {"p50": round(float(np.percentile(done, 50)), 1),
                       "p99": round(float(np.percentile(done, 99)), 1)},
        "gsamples_per_s": round(units / (queue_ms / 1e3) / 1e9, 2),
        "sequential_plain": {"value": round(n / (seq_done[-1] / 1e3), 4), "unit": "ensembles/s",
                             "ms_per_queue": round(float(seq_done[-1]), 1),
                             "latency_ms": {"p50": round(float(np.percentile(seq_done, 50)), 1),
                                            "p99": round(float(np.percentile(seq_done, 99)), 1)}},
        "power_rel_l2_batch_vs_sequential_max": worst,
        "autotune": {**choice, "seconds": round(tune_s, 2)},
        "launches": "per method either one persistent kernel (own register budget) or the single-ensemble "
                    "kernels launched per ensemble, as the autotuner measured faster; methods one after another "
                    "on one stream, one CUDA graph",
        "mode_by_method": {p.ensembles[0].method: ("per-ensemble grids" if p.ctas_per_sm == 0
                                                   else f"persistent, {p.ctas_per_sm} CTAs/SM")
                           for p in queue.parts},
        "latency_definition": "completion time since the queue started (device global timer for the persistent "
                              "kernel, CUDA events for sequential launches)",
        "dtype": "f32 math on c64 packed IQ (float64 geometry)", "data": "synthetic seeded complex Gaussian channels",
        "config": {"workload": f"{n} ensembles: depth {{128,192,256,384}} at {args.lateral} x depth x {args.lateral} "
                               "(central block of the 128-wide grid), frames {50,100,200,400}, 128 ch, "
                               "angles {5,7,11}, ns 512, 50% OPW / 25% XDoppler / 25% DMAS-CCF-ACF",
                   "seed": args.seed, "ensembles": shapes},
        "clocks": clocks, "gpu_launches": steps * sum(p.kernel_launches() for p in queue.parts),
    }


# ------------------------------------------------------ precision form --
def run_precision(args) -> dict:
    """Casorati 4,194,304 x 400 complex64 clutter scene: Gram in float64 / float32 CUDA cores and
    TF32 / 3xBF16 tensor cores, float64 EVD and projection; errors against the float64 Gram."""
    import torch

    from rcabeam_b200 import _lib, gpu_clutter, scenes

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rows, frames = args.rows, args.casorati_frames
    gen = torch.Generator(device=dev).manual_seed(args.seed)
    iq = scenes.clutter_casorati(rows, frames, generator=gen, device=dev)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    gram = gpu_clutter.Gram(frames, dev)
    out, ref_pd, ref_iq = {}, None, None
    for precision in ("complex128", "complex64", "tf32", "bf16x3"):
        for _ in range(max(1, args.warmup)):
            gram.accumulate((iq,), precision)
        torch.cuda.synchronize()
        start.record()
        for _ in range(max(1, args.steps)):
            gram.accumulate((iq,), precision)
        stop.record()
        torch.cuda.synchronize()
        gram_ms = start.elapsed_time(stop) / max(1, args.steps)
        start.record()
        _, basis = gpu_clutter.temporal_basis(iq, precision=precision)
        stop.record()
        torch.cuda.synchronize()
        basis_ms = start.elapsed_time(stop)
        start.record()
        pd = gpu_clutter.filtered_power(iq, basis, rank_start=3)
        stop.record()
        torch.cuda.synchronize()
        power_ms = start.elapsed_time(stop)
        filtered = gpu_clutter.apply_temporal_filter(iq, basis, rank_start=3)
        entry = {"gram_ms": round(gram_ms, 2), "basis_ms_incl_gram_evd": round(basis_ms, 2),
                 "filtered_power_ms": round(power_ms, 2),
                 "gram_tflops_upper": round(4 * rows * frames * (frames + 64) / gram_ms / 1e9, 1)}
        if precision == "complex128":
            ref_pd, ref_iq = pd, filtered
        else:
            entry["filtered_pd_rel_l2_vs_f64"] = float(torch.linalg.vector_norm(pd - ref_pd)
                                                       / torch.linalg.vector_norm(ref_pd))
            entry["filtered_iq_rel_l2_vs_f64"] = float(torch.linalg.vector_norm((filtered - ref_iq).abs())
                                                       / torch.linalg.vector_norm(ref_iq.abs()))
        out[precision] = entry
        del filtered
        torch.cuda.empty_cache()
    assert _lib.device_error() == 0
    return {"form": "precision", "metric": "Gram ms (Casorati rows x frames, complex64)", "forms": out,
            "reference": "float64 CUDA-core Gram + float64 EVD + float64 projection on the GPU (pinned to the "
                         "NumPy complex128 oracle in tests)",
            "config": {"workload": f"clutter scene Casorati {rows} x {frames} c64 (rank-3 tissue 0/-6/-12 dB, "
                                   "blood -40 dB in 2 % of rows, noise -50 dB), rank_start=3", "seed": args.seed},
            "data": "synthetic seeded scene model", "gpu_launches": None}


# ------------------------------------------------------ channel domain --
def run_channel(args) -> dict:
    """Channel-domain filtered OPW PD on the full workload (reference clutter_pipeline.py:85-123 with
    domain="channel"): one basis over the RC + CR channel Casorati rows (2 x 720,896 x 200), both
    apertures filtered, packed and beamformed to power (no IQ ensemble stored)."""
    import torch

    from rcabeam_b200 import _lib, pipeline
    from rcabeam_b200.sim import RCAGeometry

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    el, angles, grid = workload()
    geom = RCAGeometry(el, el, c=C, fs=FS, f_demod=FD, fnumber=None)
    gen = torch.Generator(device=dev).manual_seed(1234)
    rc, cr = pipeline.synthetic_channels((NS, NC, NA, NT), generator=gen, device=dev)
    units = units_per_step()
    results, powers = {}, {}
    for name in ("chosen", "plain"):
        storage, precision = FORMS[name]
        plan = pipeline.FilteredOpw((NS, NC, NA, NT), angles, T_START, grid, geom, rank_start=RANK_START,
                                    precision=precision, iq_storage=storage, domain="channel")
        steps = args.steps if name == "chosen" else max(1, min(args.steps, 2))
        elapsed, das_s, stages = _time_form(plan, rc, cr, steps, args.warmup if name == "chosen" else 1, 1)
        powers[name] = plan.power.clone()
        results[name] = {"ms_per_ensemble": round(elapsed / steps * 1e3, 3), "steps": steps,
                         "gsamples_per_s": round(units * steps / elapsed / 1e9, 3), "das_ms": round(das_s * 1e3, 3),
                         "stages_ms": stages, "iq_storage": storage, "gram_precision": precision,
                         "gpu_launches_per_step": plan.launches_per_step()}
        del plan
        torch.cuda.empty_cache()
    assert _lib.device_error() == 0
    ref = powers["plain"]
    return {"form": "channel", "metric": "channel-domain filtered PD ms/ensemble", "unit": "ms",
            "higher_is_better": False, "value": results["chosen"]["ms_per_ensemble"], "forms": results,
            "accuracy": {"chosen_vs_plain_filtered_pd_rel_l2": float(torch.linalg.vector_norm(powers["chosen"] - ref)
                                                                     / torch.linalg.vector_norm(ref))},
            "config": {**CONFIG, "domain": "channel"}, "data": "synthetic seeded channel IQ (complex Gaussian)"}


# ------------------------------------------------------------- St-SW --
def run_stsw(args) -> dict:
    """St-SW (method 4, k = 2, 3, 4) through the C ABI on resident channels of the full shape
    (512 x 128 x 11 x 200) over a central block of the full grid (default 32 x 64 x 32)."""
    import torch

    from rcabeam_b200 import _cuda_impl, _lib, pipeline
    from rcabeam_b200.sim import scan_coords

    global SUBGRID
    SUBGRID = tuple(args.subgrid) if args.subgrid else (32, 64, 32)
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    el, angles, grid = workload()
    gen = torch.Generator(device=dev).manual_seed(1234)
    rc, cr = pipeline.synthetic_channels((NS, NC, NA, NT), generator=gen, device=dev)
    scan = scan_coords(grid)
    nv = len(scan)
    f32 = lambda v: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)).to(dev)  # noqa: E731
    d_scan, d_el, d_ang = f32(scan), f32(el), f32(angles)
    d_starts = f32(np.full(NA, T_START))
    pd = torch.empty((nv, 2), dtype=torch.float32, device=dev)
    weights = torch.empty(nv, dtype=torch.float32, device=dev)
    units = nv * 2 * NC * NA * NT
    out = {}
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in (2, 3, 4):
        def step():
            _cuda_impl.ensemble_from_channels(rc, cr, d_scan, d_el, d_el, d_ang, d_starts, pd, None, weights, C, FS,
                                              FD, -1.0, 4, k, False)
        for _ in range(max(1, args.warmup)):
            step()
        torch.cuda.synchronize()
        start.record()
        for _ in range(max(1, args.steps)):
            step()
        stop.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(stop) / max(1, args.steps)
        out[f"k{k}"] = {"ms": round(ms, 2), "gsamples_per_s": round(units / ms / 1e6, 1)}
    assert _lib.device_error() == 0
    return {"form": "stsw", "metric": "St-SW Gsamples/s (vox*ch*ang*frm)", "unit": "Gsamples/s",
            "value": out["k2"]["gsamples_per_s"], "forms": out,
            "config": {"workload": f"St-SW on a {list(SUBGRID)} block of the full grid, channels "
                                   f"{NS}x{NC}x{NA}x{NT} c64 per aperture, full aperture", "voxels": nv,
                       "note": "timed region: pack both apertures + series kernel + finish per voxel tile"},
            "data": "synthetic seeded channel IQ (complex Gaussian)"}


# ------------------------------------------------ differentiation form --
def run_differentiation(args) -> dict:
    """Grid 64 x 128 x 64, channels (384, 128, 7, 32): forward PD of the whole grid and the
    backward of the 1 mm ROI loss through the hand-written adjoint, complex64 channels."""
    import torch

    from rcabeam_b200 import _lib
    from rcabeam_b200.autograd import DasGeometry, OpwPowerDoppler
    from rcabeam_b200.sim import RCAGeometry, scan_coords, simulate_point

    torch.cuda.set_device(0)
    ns, nc, na, nt = 384, 128, 7, 32
    el = (np.arange(nc) - (nc - 1) / 2) * PITCH
    half = (nc - 1) / 2 * PITCH
    geom = RCAGeometry(el, el, c=C, fs=FS, f_demod=FD, fnumber=None)
    angles = np.deg2rad(np.linspace(-10, 10, na))
    target = (0.35e-3, 8.0e-3, -0.22e-3)
    rng = np.random.default_rng(args.seed)
    phases = np.exp(2j * np.pi * rng.random(nt))
    chans = []
    for config in ("RC", "CR"):
        data = simulate_point(geom, angles, target, ns, T_START, config)
        noise = 0.01 * (rng.normal(size=(ns, nc, na, nt)) + 1j * rng.normal(size=(ns, nc, na, nt)))
        chans.append(torch.from_numpy((data[..., None] * phases + noise).astype(np.complex64)).cuda())
    grid = (np.linspace(-half, half, 64), np.linspace(4e-3, 12e-3, 128), np.linspace(-half, half, 64))
    geometry = DasGeometry.build(grid, geom, angles, T_START)
    scan = scan_coords(grid)
    roi = torch.from_numpy((np.sum((scan - np.array(target)) ** 2, axis=1) <= 1e-6).astype(np.float64)).cuda()
    offsets = torch.from_numpy(rng.normal(scale=5e-9, size=(2, nc))).cuda()
    rc = chans[0].requires_grad_()
    off = offsets.clone().requires_grad_()
    c = torch.tensor(1523.0, dtype=torch.float64, device="cuda", requires_grad=True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd, bwd = [], []
    for step in range(max(1, args.warmup) + max(1, args.steps)):
        rc.grad = off.grad = c.grad = None
        ev[0].record()
        pd = OpwPowerDoppler.apply(rc, chans[1], off, c, geometry, 8)
        loss = (pd * roi).sum()
        ev[1].record()
        loss.backward()
        ev[2].record()
        torch.cuda.synchronize()
        if step >= max(1, args.warmup):
            fwd.append(ev[0].elapsed_time(ev[1]))
            bwd.append(ev[1].elapsed_time(ev[2]))
    assert _lib.device_error() == 0
    units = geometry.voxels * 2 * nc * na * nt
    roi_units = int(roi.sum().item()) * 2 * nc * na * nt
    f_ms, b_ms = statistics.median(fwd), statistics.median(bwd)
    return {"form": "differentiation", "metric": "forward Gsamples/s (whole grid) and backward ms (ROI loss)",
            "forward_ms": round(f_ms, 2), "forward_gsamples_per_s": round(units / f_ms / 1e6, 1),
            "backward_ms": round(b_ms, 2), "roi_voxels": int(roi.sum().item()),
            "backward_gsamples_per_s": round(2 * roi_units / b_ms / 1e6, 2),
            "note": "backward recomputes the ROI IQ (forward units) and scatters the adjoint (same units again)",
            "dtype": "complex64 channels, float32 interpolation, float64 geometry and gradient sums",
            "config": {"workload": "grid 64x128x64 over +-7 mm x 4-12 mm, channels (384,128,7,32), point target, "
                                   "loss = sum PD over a 1 mm sphere, offsets N(0, 5 ns), c = 1523 m/s",
                       "seed": args.seed},
            "data": "simulated point target + noise"}


# ------------------------------------------------------- CPU (oracle) arms --
def _oracle_sample(seed: int, voxels: int):
    """A bounded slice of the workload for the float64 CPU oracle: voxels spread over the grid."""
    from oracle import das

    el, angles, grid = workload()
    rng = np.random.default_rng(seed)
    shape = (NS, NC, NA, NT)
    rc = (rng.standard_normal(shape, dtype=np.float32) + 1j * rng.standard_normal(shape, dtype=np.float32))
    cr = (rng.standard_normal(shape, dtype=np.float32) + 1j * rng.standard_normal(shape, dtype=np.float32))
    scan = das.scan_coords(grid).astype(np.float64)
    ids = np.unique(np.linspace(0, len(scan) - 1, voxels).round().astype(np.int64))
    return rc.astype(np.complex64), cr.astype(np.complex64), scan[ids], el, angles


_SHARED = {}


def _attach(names, shape, el, angles):
    """Pool initializer: map the parent's channel arrays (shared memory, no copies)."""
    from multiprocessing import shared_memory

    for key, name in names.items():
        block = shared_memory.SharedMemory(name=name)
        _SHARED[key + "_block"] = block
        _SHARED[key] = np.ndarray(shape, dtype=np.complex64, buffer=block.buf)
    _SHARED["el"], _SHARED["angles"] = el, angles


def _oracle_chunk(scan):
    from oracle import das

    return das.opw_iq(_SHARED["rc"], _SHARED["cr"], scan, _SHARED["el"], _SHARED["el"], _SHARED["angles"], T_START,
                      C, FS, FD, None)


def cpu_baseline(args, voxels_per_core: int) -> dict:
    """Time the float64 NumPy restatement of the reference's CPU path on a bounded voxel sample, on
    every host core: DAS + OPW of the sample (reference sim._delay_numpy / opw.py), then the Gram
    clutter filter over the sample's rows and the filtered power (clutter.py:74-109, power.py).

    The channels live in shared memory that every worker maps; the spawn pool is started
    before the timed region.  The sample is the same fraction of every stage's work (all
    stages are linear in the voxel count), so units / seconds is the path's rate."""
    import multiprocessing as mp
    from multiprocessing import shared_memory

    from oracle import clutter as oc

    cores = os.cpu_count() or 1
    voxels = voxels_per_core * cores
    rc, cr, scan, el, angles = _oracle_sample(7, voxels)
    voxels = len(scan)
    blocks = {}
    try:
        for key, arr in (("rc", rc), ("cr", cr)):
            blocks[key] = shared_memory.SharedMemory(create=True, size=arr.nbytes)
            np.ndarray(arr.shape, dtype=np.complex64, buffer=blocks[key].buf)[...] = arr
        names = {k: b.name for k, b in blocks.items()}
        chunks = np.array_split(scan, cores)
        with mp.get_context("spawn").Pool(cores, initializer=_attach, initargs=(names, rc.shape, el, angles)) as pool:
            pool.map(len, [[0]] * cores)  # workers started and attached
            begin = time.perf_counter()
            iq = np.concatenate(pool.map(_oracle_chunk, chunks))
            _, basis = oc.temporal_basis(iq, method="gram")
            oc.filtered_power(iq, basis, RANK_START)
            seconds = time.perf_counter() - begin
    finally:
        for b in blocks.values():
            b.close()
            b.unlink()
    units = voxels * 2 * NC * NA * NT
    return {"value": round(units / seconds / 1e9, 5), "unit": "Gsamples/s", "cores": cores, "kind": "port",
            "sample": f"{voxels} voxels spread over the grid x 256 ch x 11 ang x 200 frm of the workload: DAS + OPW "
                      "(float64 NumPy restatement of reference sim._delay_numpy), Gram clutter filter over the "
                      f"sample rows and filtered PD (restatement of clutter.py:74-109), {seconds:.1f} s"}


def run_reference(args, rank: int, world: int) -> dict | None:
    """The reference arm: the float64 NumPy restatement of the reference's CPU path, one bounded
    sample per step on all host cores (rank 0 only)."""
    if rank != 0:
        return None
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(args, voxels_per_core=args.reference_voxels)
    for _ in range(args.steps):
        vals.append(cpu_baseline(args, voxels_per_core=args.reference_voxels))
    value = statistics.median(v["value"] for v in vals)
    base = dict(vals[-1])
    base["value"] = value
    return {
        "impl": "reference", "metric": "OPW Gsamples/s (vox*ch*ang*frm), filtered PD", "value": value,
        "unit": "Gsamples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": CONFIG, "cpu_baseline": base,
        "e2e": {"value": value, "unit": "Gsamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-voxels", type=int, default=768,
                    help="oracle voxels per core for the CPU baseline of the B200 line (~10 s)")
    ap.add_argument("--reference-voxels", type=int, default=192,
                    help="oracle voxels per core per step of the reference arm (~3 s per step)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the float64 oracle sample (profiling runs)")
    ap.add_argument("--only-chosen", action="store_true", help="time only the chosen form (profiling runs)")
    ap.add_argument("--grid", type=int, nargs=3, default=None, metavar=("NX", "NZ", "NY"),
                    help="reduced grid for profiling runs (the reported workload is the default)")
    ap.add_argument("--frames", type=int, default=None, help="reduced frame count for profiling runs")
    ap.add_argument("--channels", type=int, default=None, help="reduced channel count for profiling runs")
    ap.add_argument("--subgrid", type=int, nargs=3, default=None, metavar=("NX", "NZ", "NY"),
                    help="central block of the full grid at full resolution (profiling runs)")
    ap.add_argument("--form", default="filtered",
                    choices=["filtered", "batching", "precision", "differentiation", "channel", "stsw"],
                    help="filtered: the filtered-OPW headline; batching, precision, differentiation: the forms")
    ap.add_argument("--rows", type=int, default=128 * 256 * 128, help="Casorati rows of the precision form")
    ap.add_argument("--casorati-frames", type=int, default=400, help="Casorati frames of the precision form")
    ap.add_argument("--ensembles", type=int, default=48, help="queue length of the batching form")
    ap.add_argument("--seed", type=int, default=5, help="seed of the batching queue")
    ap.add_argument("--lateral", type=int, default=128,
                    help="lateral x / y points of the batching queue's grids (central block of 128)")
    args = ap.parse_args()
    if args.form != "filtered":
        if args.impl == "b200" and int(os.environ.get("RANK", "0")) == 0:
            run = {"batching": run_batching, "precision": run_precision, "differentiation": run_differentiation,
                   "channel": run_channel, "stsw": run_stsw}
            print(json.dumps(run[args.form](args)), flush=True)
        return
    global GRID_SHAPE, NT, NC, SUBGRID
    if args.subgrid:
        SUBGRID = tuple(args.subgrid)
        CONFIG["grid"] = list(SUBGRID)
        CONFIG["workload"] += f" (REDUCED to the central {SUBGRID} block for profiling)"
    if args.channels:
        NC = args.channels
        CONFIG["channels"] = NC
        CONFIG["workload"] += f" (REDUCED to {NC} channels for profiling)"
    if args.frames:
        NT = args.frames
        CONFIG["frames"] = NT
        CONFIG["workload"] += f" (REDUCED to {NT} frames for profiling)"
    if args.grid:
        GRID_SHAPE = tuple(args.grid)
        CONFIG["grid"] = list(GRID_SHAPE)
        CONFIG["workload"] += f" (REDUCED grid {GRID_SHAPE} for profiling)"
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        if world > 1:
            import datetime

            import torch

            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        line = run_b200(args, rank, world)
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
