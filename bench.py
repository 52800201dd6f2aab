"""Benchmark: the 324-tree 1920x1080 forest walk (1 spp, sun shadows off).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl arbor|reference]
                    [--workload forest|shadows|wind|tree|batch|denoise|species] [--no-cpu-baseline]
                    [--no-target]

A step is one frame of the seeded 64-frame walk: updateCamera, tracePixels,
shadePixels and filterLighting+resolvePixels over 1920x1080 pixels, on a
scene (master seed 7) built once.  `value` is primary rays per second of the
whole job (all ranks) with inputs resident on the device; `e2e` is the same
metric through the engine API with the input record copied from pinned host
memory and the RGBA8 frame copied back to the host every step.  The default
forest run then measures the same walk with tree-to-tree sun shadows on (the
target configuration) and reports it, with its own CPU baseline, under
`target_shadows`.

Multi-GPU: the path shards by frames/pixels with no exchange, so each rank
renders its own frames (weak scaling, replicas); timing is the max over ranks.

--impl reference times the reference's own CPU implementation (the harness
code built from the reference's sources, oracle/_ref; the oracle port when
that build is absent) on a band of rows of the same frame, on all host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "arbor-cuda_b200"))

import numpy as np  # noqa: E402

METRIC = "1080p forest ms/frame & Mrays/s; learned vs filterLighting ms at equal PSNR"
UNIT = "Mrays/s"
WALK_FRAMES = 64


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="arbor", choices=["arbor", "reference"])
    ap.add_argument("--workload", default="forest", choices=["forest", "shadows", "wind", "tree", "batch", "denoise", "species"])
    ap.add_argument("--species", type=int, default=16, help="species workload: distinct trees (scenes) in the forest")
    ap.add_argument("--views", type=int, default=64, help="batch workload: views per batch")
    ap.add_argument("--scenes", type=int, default=16, help="batch workload: resident scenes (master seeds)")
    ap.add_argument("--tune-views", type=int, default=8, help="batch workload: views the autotuner times each configuration on")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    ap.add_argument("--width", type=int, default=0, help="override the workload's width (profiling runs)")
    ap.add_argument("--height", type=int, default=0, help="override the workload's height (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the engine-API end-to-end leg (profiling runs)")
    ap.add_argument("--no-target", action="store_true",
                    help="forest workload: skip the second measurement of the same walk with sun shadows on (target_shadows)")
    return ap.parse_args()


def workload_spec(name: str) -> dict:
    base = {"seed": 7, "width": 1920, "height": 1080, "spp": 1, "shadows": False, "single_tree": False, "wind": False, "rebuild": False}
    if name == "forest":
        return {**base, "workload": "forest-1080p-walk: 324-tree forest from master seed 7, 1920x1080, 1 spp, sun shadows off, "
                                    "64-frame seeded walk at 1.4 m/s, eye height 1.72 m"}
    if name == "shadows":
        return {**base, "shadows": True,
                "workload": "forest-1080p-walk-shadows: the forest walk with tree-to-tree sun shadows on "
                            "(sun elevation 35 deg, azimuth from the seed)"}
    if name == "species":
        return {**base, "species": 16,
                "workload": "forest-1080p-walk-species: the forest walk (shadows off) with 16 species: instance t takes its own records and "
                            "BVH from the scene of seed s[forestSeed(t, 7) mod 16] (seeds 7 and seeded draws), 16 scenes resident"}
    if name == "wind":
        return {**base, "shadows": True, "wind": True, "rebuild": True, "spp": 4,
                "workload": "forest-1080p-wind: the forest walk at 4 spp per frame, sun shadows on (35 deg, azimuth from the seed), "
                            "wind-animated leaves, scene and BVH rebuilt every frame"}
    return {**base, "seed": 1, "width": 256, "height": 256, "single_tree": True,
            "workload": "tree-256: one tree from master seed 1, 256x256, 1 spp, 6 m camera, 60 deg FOV, shadows off"}


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def physical_gpu(local_rank: int) -> str:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return str(local_rank)


# -------------------------------------------------------------- arbor arm --
class Frames:
    """Device buffers and the per-frame launch sequence through the C-ABI."""

    def __init__(self, ab, spec: dict, torch):
        self.ab, self.torch, self.spec = ab, torch, spec
        w, h = spec["width"], spec["height"]
        self.w, self.h = w, h
        f32 = lambda n: torch.zeros(n, dtype=torch.float32, device="cuda")  # noqa: E731
        i32 = lambda n: torch.zeros(n, dtype=torch.int32, device="cuda")  # noqa: E731
        import workloads

        ns = spec.get("species", 1)
        self.B, self.P, self.Keys, self.Order, self.Nodes = (f32(2109 * 20), f32(ns * 32768 * 24), i32(ns * 32768), i32(ns * 32768),
                                                             f32(ns * 65536 * 8))
        self.C = f32(64)
        self.scratch = i32(2 * 32768)
        self.Hit, self.Lin, self.Gui, self.Fil, self.Hist = (f32(w * h * 4) for _ in range(5))
        self.Pix = i32(w * h)
        self.species = None
        if ns > 1:
            # one scene per species seed, back to back; species 0 is the master seed
            self.seeds = workloads.batch_seeds(ns, spec["seed"])
            for k, sd in enumerate(self.seeds):
                self.B.zero_()
                sl = lambda t, n: t[k * n:(k + 1) * n]  # noqa: E731
                self.check(ab.call("arbor_buildScene", sd, self.B, sl(self.P, 32768 * 24), sl(self.Keys, 32768), sl(self.Order, 32768),
                                   sl(self.Nodes, 65536 * 8), self.C if k == 0 else None, self.scratch))
            import ctypes

            self.of = np.ascontiguousarray(workloads.species_of(ns, spec["seed"]), np.int32)
            self.species = (ns, self.of.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        else:
            self.check(ab.call("arbor_buildScene", spec["seed"], self.B, self.P, self.Keys, self.Order, self.Nodes, self.C, self.scratch))

        if spec["single_tree"]:
            self.C.copy_(torch.from_numpy(workloads.single_tree_camera(w, h, spec["seed"])))
        else:
            self.C.copy_(torch.from_numpy(workload_state(self.C.cpu().numpy(), spec)))
        inputs = np.zeros((WALK_FRAMES, 32), np.float32)
        self.dts = []
        for k in range(WALK_FRAMES):
            inputs[k], dt = workloads.walk_input(k, spec["seed"])
            self.dts.append(dt)
        self.I = torch.from_numpy(inputs).cuda()
        self.trace = "arbor_traceTreePixels" if spec["single_tree"] else "arbor_tracePixels"
        self.shade = "arbor_shadeTreePixels" if spec["single_tree"] else "arbor_shadePixels"
        torch.cuda.synchronize()

    def check(self, st):
        if st != self.ab.OK:
            raise RuntimeError(f"{self.ab.STATUS.get(st)}: {self.ab.last_error()}")

    def build(self):
        """The per-frame scene rebuild (camera record untouched)."""
        self.check(self.ab.call("arbor_buildScene", self.spec["seed"], self.B, self.P, self.Keys, self.Order, self.Nodes, None, self.scratch))

    def trace_call(self):
        if self.species:
            return self.ab.call("arbor_traceSpeciesPixels", self.P, self.Nodes, self.Order, *self.species, self.C, self.Hit, self.w, self.h)
        return self.ab.call(self.trace, self.P, self.Nodes, self.Order, self.C, self.Hit, self.w, self.h)

    def shade_call(self):
        if self.species:
            return self.ab.call("arbor_shadeSpeciesPixels", self.P, self.Nodes, self.Order, *self.species, self.C, self.Hit, self.Lin, self.Gui,
                                self.w, self.h)
        return self.ab.call(self.shade, self.P, self.Nodes, self.Order, self.C, self.Hit, self.Lin, self.Gui, self.w, self.h)

    def sample(self):
        ab, w, h = self.ab, self.w, self.h
        self.check(self.trace_call())
        self.check(self.shade_call())
        self.check(ab.call("arbor_filterResolve", self.Lin, self.Gui, self.Hit, self.Fil, self.Hist, self.Pix, self.C, w, h))

    def step(self, k: int):
        ab, w, h = self.ab, self.w, self.h
        if self.spec["rebuild"]:
            self.build()
        if not self.spec["single_tree"]:
            Ik = self.I[k % WALK_FRAMES]
            self.check(ab.call("arbor_updateCamera", self.C, Ik, self.P, self.dts[k % WALK_FRAMES], w, h))
        spp = self.spec["spp"]
        for s in range(spp):
            if spp > 1:
                # progressive samples of one frame, as the harness's render loop
                # sets C[9] and C[10] (tests/native_harness.cpp:62)
                self.check(ab.call("arbor_setSample", self.C, s, int(s == 0)))
            self.sample()


def workload_state(C: np.ndarray, spec: dict) -> np.ndarray:
    """The camera/state record of a forest workload on top of initCamera's."""
    import workloads

    C = C.copy()
    C[22] = 1.0 if spec["shadows"] else 0.0
    if spec["shadows"]:
        C[12], C[13] = workloads.shadow_sun(spec["seed"])
    if spec.get("wind"):
        C[11] = 0.60  # the breeze toggle's amplitude (Arbor.cu:182)
    return C


# Algorithmic bytes of one scene build: makeKeys 32768 x (96 + 8), the sort
# 16 B per element per pass x 4 passes, makeBounds 32768 x (4 + 96 + 32),
# the reduce levels 32767 x 96 (Arbor.cu:139-142).
BUILD_BYTES = 32768 * (96 + 8) + 16 * 32768 * 4 + 32768 * (4 + 96 + 32) + 32767 * 96


def max_over_ranks(ms: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's time (every rank calls it; a no-op for one rank)."""
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    return float(t.item())


def replica_rate(units_per_rank_step: float, steps: int, ms_max: float, world: int) -> float:
    """Whole-job rate in millions of units per second: every rank (a replica)
    processed units_per_rank_step per step, the job took ms_max."""
    return world * units_per_rank_step * steps / (ms_max / 1e3) / 1e6


def time_kernel(torch, fn, reps: int) -> float:
    """Mean ms per call of fn() with CUDA events on the current stream."""
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) / reps


# Used when MEASURED_PEAKS.json is absent: an earlier measurement on B200s of
# this pool (STREAM-style copy, cuBLAS BF16 GEMM burst).
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh) | {"source": "measured"}
    except (OSError, ValueError):
        return dict(FALLBACK_PEAKS)


def run_arbor(args, rank: int, world: int, local_rank: int) -> None:
    spec = workload_spec(args.workload)
    if args.width and args.height:
        spec.update(width=args.width, height=args.height, workload=spec["workload"] + f" (at {args.width}x{args.height})")
    if args.workload == "species":
        spec["species"] = args.species
    result = measure_workload(args, spec, rank, world, local_rank)
    if args.workload == "forest" and not args.no_target:
        # The target configuration: the same walk with tree-to-tree sun
        # shadows on, measured the same way, with its own CPU baseline.
        tspec = workload_spec("shadows")
        if args.width and args.height:
            tspec.update(width=args.width, height=args.height, workload=tspec["workload"] + f" (at {args.width}x{args.height})")
        t = measure_workload(args, tspec, rank, world, local_rank)
        keep = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "config", "phases_ms", "roofline", "roofline_trace",
                "roofline_shade", "roofline_hbm", "gpu_launches", "clocks", "e2e", "cpu_baseline")
        result["target_shadows"] = {k: t[k] for k in keep if k in t}
        cpu = t.get("cpu_baseline", {}).get("value")
        e2e = (t.get("e2e") or {}).get("value")
        if cpu and e2e:
            result["target_shadows"]["e2e_over_cpu_baseline"] = round(e2e / cpu, 1)
        result["gpu_launches"] += t["gpu_launches"]
    if rank == 0:
        print(json.dumps(result), flush=True)


def measure_workload(args, spec: dict, rank: int, world: int, local_rank: int) -> dict:
    """Time `args.steps` frames of one workload (after `args.warmup`) and
    return its JSON record (every rank calls it; max over ranks)."""
    import torch
    import torch.distributed as dist

    import arbor_b200 as ab

    fr = Frames(ab, spec, torch)
    w, h = fr.w, fr.h
    for k in range(args.warmup):
        fr.step(k)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(physical_gpu(local_rank))
    sampler.start()
    time.sleep(0.3)
    launches0 = ab.launches()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for k in range(args.steps):
        fr.step(args.warmup + k)
    end.record()
    end.synchronize()
    torch.cuda.synchronize()
    launches = ab.launches() - launches0
    clocks = sampler.stop()
    ms_max = max_over_ranks(start.elapsed_time(end), world)
    ms_per_step = ms_max / args.steps
    rays_per_step = w * h * spec["spp"]
    value = replica_rate(rays_per_step, args.steps, ms_max, world)

    # Per-kernel durations (same stream, CUDA events, after the timed region).
    k0 = args.warmup + args.steps
    fr.step(k0)
    reps = 8
    ms_trace = time_kernel(torch, lambda: fr.check(fr.trace_call()), reps)
    ms_shade = time_kernel(torch, lambda: fr.check(fr.shade_call()), reps)
    ms_fr = time_kernel(torch, lambda: fr.check(ab.call("arbor_filterResolve", fr.Lin, fr.Gui, fr.Hit, fr.Fil, fr.Hist, fr.Pix, fr.C, w, h)), reps * 4)
    ms_build = time_kernel(torch, fr.build, reps * 4) if not fr.species else None
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs")
    hbm_source = "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks["source"] == "measured" else "6650 GB/s (of fallback)"
    # filterLighting+resolvePixels algorithmic bytes per pixel: Linear, Guide,
    # Hit read (48) + Filtered write (16) + History read+write (32, History
    # read only when the sample count is non-zero) + Pixels write (4).
    count_nonzero = float(fr.C[9].item()) >= 0.5 and float(fr.C[10].item()) <= 0.5
    fr_bytes = w * h * (48 + 16 + (32 if count_nonzero else 16) + 4)
    fr_gbs = fr_bytes / (ms_fr / 1e3) / 1e9
    sm_clock = clocks.get("sm_mhz") or peaks.get("clocks_under_load", {}).get("sm_mhz_median") or 1965.0
    fp32_peak = 148 * 128 * sm_clock * 1e6 / 1e12  # one non-fused FP32 op per lane per cycle, TOP/s

    result = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: procedural scene grown from the master seed; seeded camera walk (no dataset)",
        "config": {**{k: v for k, v in spec.items()}, "frames_in_walk": WALK_FRAMES, "parallelism": f"replicas x{world}",
                   "l2": "per-step frame buffers (Hit, Linear, Guide, Filtered, History, Pixels = 174 MB at 1080p) exceed the "
                         "126 MB L2; the 5.7 MB scene stays resident by design"},
        "phases_ms": {"trace": round(ms_trace, 4), "shade": round(ms_shade, 4), "filter_resolve": round(ms_fr, 4),
                      "build": round(ms_build, 4) if ms_build else None, "per_sample": ["trace", "shade", "filter_resolve"],
                      "per_frame": (["build"] if spec["rebuild"] else []) + ["update_camera"] + (["set_sample"] if spec["spp"] > 1 else [])},
        "roofline": None,
        "roofline_hbm": {"kernel": "filterResolve", "bound": "hbm", "achieved": round(fr_gbs, 1), "peak": hbm_peak, "unit": "GB/s",
                         "frac": round(fr_gbs / hbm_peak, 4) if hbm_peak else None, "traffic": None,
                         "algorithmic_bytes": fr_bytes, "peak_source": hbm_source},
        "roofline_build": None if not ms_build else {
            "kernel": "buildScene (growth, primitives + keys, 4 radix passes, bounds)", "bound": "hbm",
            "achieved": round(BUILD_BYTES / (ms_build / 1e3) / 1e9, 1), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(BUILD_BYTES / (ms_build / 1e3) / 1e9 / hbm_peak, 4) if hbm_peak else None, "traffic": None,
            "algorithmic_bytes": BUILD_BYTES, "ms_per_build": round(ms_build, 4),
            "note": "13 MB over a few dependent launches of a few thousand threads: launch- and latency-bound, far "
                    "from the HBM roof", "peak_source": hbm_source},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    import roofline_model

    # The FP32 roofline of the dominant kernel (trace, or shade when sun
    # shadows make it the longer pass); both are reported.
    if fr.species:
        # the work counter runs one scene; no FP32 count for a forest of several species
        result["roofline"] = result["roofline_hbm"]
    else:
        result["roofline_trace"] = roofline_model.trace_roofline(ab, fr, torch, ms_trace, fp32_peak, sm_clock)
        result["roofline_shade"] = roofline_model.shade_roofline(ab, fr, torch, ms_shade, fp32_peak, sm_clock)
        result["roofline"] = result["roofline_trace"] if ms_trace >= ms_shade else result["roofline_shade"]

    # End to end through the engine API with host buffers.
    if not args.no_e2e:
        if fr.species:
            result["e2e"] = run_e2e_frames(ab, torch, fr, args)
        elif spec["spp"] == 1 and not spec["rebuild"]:
            result["e2e"] = run_e2e(ab, torch, spec, args)
        else:
            result["e2e"] = {"value": None, "unit": UNIT, "note": "the engine API renders one sample per frame without rebuilds"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_species_sample(fr, args.cpu_seconds) if fr.species else cpu_baseline(spec, args.cpu_seconds)
    del fr
    return result


def run_e2e_frames(ab, torch, fr, args) -> dict:
    """End to end through the C-ABI entries: every step copies the frame's
    input record from pinned host memory, runs the frame and copies the
    RGBA8 frame back to pinned host memory."""
    import workloads

    w, h = fr.w, fr.h
    stream = torch.cuda.current_stream()
    inputs = torch.from_numpy(np.stack([workloads.walk_input(k, fr.spec["seed"])[0] for k in range(WALK_FRAMES)])).pin_memory()
    I_dev = torch.zeros(32, device="cuda")
    host = torch.empty(w * h, dtype=torch.int32).pin_memory()

    def one(k):
        I_dev.copy_(inputs[k % WALK_FRAMES], non_blocking=True)
        fr.check(ab.call("arbor_updateCamera", fr.C, I_dev, fr.P, fr.dts[k % WALK_FRAMES], w, h))
        fr.sample()
        host.copy_(fr.Pix, non_blocking=True)

    for k in range(args.warmup):
        one(k)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for k in range(args.steps):
        one(args.warmup + k)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    return {"value": round(w * h * args.steps / (ms / 1e3) / 1e6, 3), "unit": UNIT, "h2d_bytes_per_step": 32 * 4,
            "d2h_bytes_per_step": w * h * 4, "ms_per_step": round(ms / args.steps, 4),
            "api": "arbor_updateCamera + arbor_traceSpeciesPixels + arbor_shadeSpeciesPixels + arbor_filterResolve (pinned host buffers)"}


def cpu_species_sample(fr, target_s: float) -> dict:
    """The oracle's forest of several species (each instance's traceTree on
    its own scene, as the reference composes traceTree per instance) on a
    band of rows of the walk's first frame."""
    o, _ = cpu_oracle()
    if not hasattr(o.lib, "oracle_tracePixelsSpecies"):
        from pyoracle import Oracle

        o = Oracle("port")
    import workloads

    spec = fr.spec
    w, h = spec["width"], spec["height"]
    scenes = [o.build_scene(sd) for sd in fr.seeds]
    C = workload_state(o.init_camera(scenes[0]["P"], spec["seed"]), spec)
    I, dt = workloads.walk_input(0, spec["seed"])
    o.update_camera(C, I, scenes[0]["P"], dt, w, h)
    rows = max(4, o.max_threads())
    y0 = h // 2 - rows // 2
    for _ in range(2):
        t0 = time.perf_counter()
        hit = o.trace_species(scenes, fr.of, C, w, h, y0, y0 + rows)
        o.shade_species(scenes, fr.of, C, hit, w, h, y0, y0 + rows)
        secs = time.perf_counter() - t0
        if secs >= target_s * 0.5 or rows >= h // 2:
            break
        rows = int(min(h // 2, max(rows, rows * target_s / max(secs, 1e-3))))
        y0 = h // 2 - rows // 2
    return {"value": round(rows * w / secs / 1e6, 4), "unit": UNIT, "cores": o.max_threads(), "kind": "port",
            "sample": f"rows {y0}..{y0 + rows - 1} of frame 0 ({rows * w} primary rays, {secs:.2f} s): trace and shade of the "
                      "oracle's forest of several species (the reference has no such forest)", "seconds": round(secs, 3)}


def run_e2e(ab, torch, spec: dict, args) -> dict:
    import workloads

    w, h = spec["width"], spec["height"]
    stream = torch.cuda.current_stream()
    eng = ab.Engine(w, h, seed=spec["seed"], single_tree=spec["single_tree"], stream=stream)
    try:
        if eng.inspect().width != w or eng.inspect().height != h:
            return {"value": None, "unit": UNIT, "note": "engine rounds this size"}
        state = np.array(eng.inspect().camera, np.float32)
        if spec["single_tree"]:
            state = workloads.single_tree_camera(w, h, spec["seed"])
        else:
            state = workload_state(state, spec)
        eng.set_state(state)
        host = torch.empty(w * h, dtype=torch.int32).pin_memory()
        n = w * h
        for k in range(args.warmup):
            I, dt = workloads.walk_input(k, spec["seed"])
            eng.set_input(I)
            eng.frame(dt)
            eng.read_pixels_into(host.data_ptr(), n)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record(stream)
        for k in range(args.steps):
            I, dt = workloads.walk_input(args.warmup + k, spec["seed"])
            eng.set_input(I)
            eng.frame(dt)
            eng.read_pixels_into(host.data_ptr(), n)
        b.record(stream)
        b.synchronize()
        wall = time.perf_counter() - t0
        ms = a.elapsed_time(b)
        value = w * h * spec["spp"] * args.steps / (ms / 1e3) / 1e6
        return {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 32 * 4, "d2h_bytes_per_step": w * h * 4,
                "ms_per_step": round(ms / args.steps, 4), "host_wall_ms_per_step": round(wall * 1e3 / args.steps, 4),
                "api": "arbor_engine_set_input + arbor_engine_frame + arbor_engine_read_pixels (pinned host buffers)"}
    finally:
        eng.close()


# ------------------------------------------------------------ CPU baseline --
def cpu_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle, available

    if available("reference"):
        return Oracle("reference"), "reference"
    return Oracle("port"), "port"


class CpuFrame:
    """The workload's first frame on the CPU implementation, rendered on an
    evenly strided subset of its rows (a representative sample of the frame;
    each pass is one OpenMP loop over the sampled rows)."""

    def __init__(self, o, spec: dict):
        import workloads

        self.o, self.spec = o, spec
        w, h, seed = spec["width"], spec["height"], spec["seed"]
        self.scene = o.build_scene(seed)
        if spec["single_tree"]:
            C = workloads.single_tree_camera(w, h, seed)
        else:
            C = workload_state(o.init_camera(self.scene["P"], seed), spec)
            I, dt = workloads.walk_input(0, seed)
            o.update_camera(C, I, self.scene["P"], dt, w, h)
        self.C = C
        self.bufs = {k: np.zeros(w * h * 4, np.float32) for k in ("Hit", "Linear", "Guide", "Filtered", "History")}
        self.bufs["Pixels"] = np.zeros(w * h, np.uint32)

    def rows(self, n: int) -> np.ndarray:
        h = self.spec["height"]
        n = max(1, min(n, h))
        return np.unique((np.arange(n) * h // n + (h // n) // 2).clip(0, h - 1)).astype(np.int32)

    def render(self, n: int) -> tuple[int, float, int]:
        rows = self.rows(n)
        spp = self.spec["spp"]
        t0 = time.perf_counter()
        for s in range(spp):
            if spp > 1:
                self.C[9], self.C[10] = s, float(s == 0)
            self.o.frame_rows(self.scene, self.C, self.spec["width"], self.spec["height"], rows, self.bufs, single=self.spec["single_tree"])
        secs = time.perf_counter() - t0
        return len(rows) * self.spec["width"] * self.spec["spp"], secs, len(rows)

    def calibrate(self, target_s: float) -> int:
        """Number of sampled rows for about target_s seconds (at least 4 per host thread)."""
        h = self.spec["height"]
        n = min(h, 4 * max(1, self.o.max_threads()))
        _, secs, n = self.render(n)
        return int(min(h, max(n, n * target_s / max(secs, 1e-3))))


def cpu_sample(o, kind: str, spec: dict, target_s: float) -> dict:
    frame = CpuFrame(o, spec)
    n = frame.calibrate(target_s)
    rays, secs, n = frame.render(n)
    return {"value": round(rays / secs / 1e6, 4), "unit": UNIT, "cores": o.max_threads(), "kind": kind,
            "sample": f"{n} evenly strided rows of {spec['height']} of frame 0 ({rays} primary rays, {secs:.2f} s): "
                      "trace, shade, filter, resolve",
            "seconds": round(secs, 3)}


def cpu_baseline(spec: dict, target_s: float) -> dict:
    o, kind = cpu_oracle()
    return cpu_sample(o, kind, spec, target_s)


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    if args.workload == "batch":
        run_reference_batch(args)
        return
    if args.workload == "species":
        run_reference_species(args)
        return
    spec = workload_spec(args.workload)
    if args.width and args.height:
        spec.update(width=args.width, height=args.height)
    o, kind = cpu_oracle()
    frame = CpuFrame(o, spec)
    # Each step renders the same evenly spaced bands, sized to about 2 s, so
    # that warmup + steps finish within a few minutes.
    n = frame.calibrate(float(os.environ.get("ARBOR_REFERENCE_STEP_SECONDS", "2.0")))
    times, rays = [], 0
    for k in range(args.warmup + args.steps):
        rays, secs, n = frame.render(n)
        if k >= args.warmup:
            times.append(secs)
    total_s = sum(times)
    value = rays * len(times) / total_s / 1e6
    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_s * 1e3 / len(times), 2), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic: procedural scene grown from the master seed", "impl": "reference",
            "config": {**spec, "sample_rows": n},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": o.max_threads(), "kind": kind,
                             "sample": f"each step renders {n} evenly strided rows of {spec['height']} of frame 0 "
                                       f"({rays} primary rays): trace, shade, filter, resolve"},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_species(args) -> None:
    """The oracle's forest of several species (no reference counterpart) on
    a band of rows per step, on all host cores."""
    import types

    import workloads

    spec = workload_spec("species")
    ns = args.species
    spec["species"] = ns
    fr = types.SimpleNamespace(spec=spec, seeds=workloads.batch_seeds(ns, spec["seed"]), of=workloads.species_of(ns, spec["seed"]))
    step_s = float(os.environ.get("ARBOR_REFERENCE_STEP_SECONDS", "2.0"))
    samples = [cpu_species_sample(fr, step_s) for _ in range(args.warmup + args.steps)][args.warmup:]
    value = statistics.mean(x["value"] for x in samples)
    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * statistics.mean(x["seconds"] for x in samples), 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic: procedural scenes grown from the species seeds", "impl": "reference",
            "config": spec, "cpu_baseline": {k: samples[-1][k] for k in ("unit", "cores", "kind", "sample")} | {"value": round(value, 4)},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ batch views --
def batch_spec(args) -> dict:
    return {"workload": f"batch-{args.views}-views: {args.views} views of {args.scenes} resident forests (324 trees each, master seeds "
                        "7 and seeded draws), resolutions uniform over 320x180/640x360/1280x720/1920x1080, seeded poses inside the "
                        "forest at 1.72 m, 1 spp, sun shadows on; one CUDA graph launch per batch",
            "views": args.views, "scenes": args.scenes, "spp": 1, "shadows": True}


def run_batch(args, rank: int, world: int, local_rank: int) -> None:
    import torch
    import torch.distributed as dist

    import arbor_b200 as ab
    import roofline_model
    import workloads

    spec = batch_spec(args)
    seeds = workloads.batch_seeds(args.scenes)
    views = workloads.batch_views(args.views, seeds)
    stream = torch.cuda.current_stream()
    b = ab.Batch(seeds, views, stream=stream)
    try:
        info = b.inspect()
        total_px = int(info.total_pixels)
        t0 = time.perf_counter()
        best, table = b.autotune(args.tune_views)
        tune_s = time.perf_counter() - t0
        for _ in range(args.warmup):
            b.render()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        sampler = ClockSampler(physical_gpu(local_rank))
        sampler.start()
        time.sleep(0.3)
        launches0 = ab.launches()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        for _ in range(args.steps):
            b.render()
        end.record()
        end.synchronize()
        launches = ab.launches() - launches0
        clocks = sampler.stop()
        ms_max = max_over_ranks(start.elapsed_time(end), world)
        value = replica_rate(total_px, args.steps, ms_max, world)

        # Per-kernel durations: the graph's kernels launched one by one.
        prof = [b.profile() for _ in range(2)][-1]
        ms_setup, ms_trace, ms_shade, ms_filter = prof
        peaks = measured_peaks()
        hbm_peak = peaks.get("hbm_gbs")
        hbm_source = "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks["source"] == "measured" else "6650 GB/s (of fallback)"
        sm_clock = clocks.get("sm_mhz") or peaks.get("clocks_under_load", {}).get("sm_mhz_median") or 1965.0
        fp32_peak = 148 * 128 * sm_clock * 1e6 / 1e12
        tc, sc = {}, {}
        for v, (_, w, h, _) in enumerate(views):
            buf = b.buffers(v)
            tc = roofline_model.add_counts(tc, roofline_model.count_events(ab, buf.P, buf.Nodes, buf.Order, buf.C, w, h, False, torch))
            sc = roofline_model.add_counts(sc, roofline_model.count_events(ab, buf.P, buf.Nodes, buf.Order, buf.C, w, h, False, torch, Hit=buf.Hit))
        r_trace = roofline_model.roofline_entry("batch trace pass (tracePixels of every view)", tc, total_px, ms_trace, fp32_peak, sm_clock)
        r_shade = roofline_model.roofline_entry("batch shade pass (shadePixels of every view)", sc, total_px, ms_shade, fp32_peak, sm_clock)
        # first sample of every view (history reset): Linear, Guide, Hit read, Filtered and History written, Pixels written
        fr_bytes = total_px * (48 + 16 + 16 + 4)
        fr_gbs = fr_bytes / (ms_filter / 1e3) / 1e9
        result = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: procedural scenes grown from the master seeds; seeded poses (no dataset)",
            "config": {**spec, "total_pixels": total_px, "parallelism": f"replicas x{world}",
                       "resolutions": {f"{w}x{h}": sum(1 for v in views if (v[1], v[2]) == (w, h)) for w, h in workloads.BATCH_RESOLUTIONS},
                       "l2": f"per-step images ({total_px * 84 / 1e9:.2f} GB) far exceed the 126 MB L2"},
            "autotune": {"chosen": best, "sample_views": args.tune_views, "seconds": round(tune_s, 2),
                         "ms_per_config": {f"tw{tw}_ctas{c}_order{o}_q{q}": round(table[i], 3)
                                           for i, (tw, c, o, q) in enumerate((tw, c, o, q) for tw in (16, 32) for c in (1, 2)
                                                                             for o in (0, 1) for q in (4, 8))}},
            "phases_ms": {"setup": round(ms_setup, 4), "trace": round(ms_trace, 4), "shade": round(ms_shade, 4),
                          "filter_resolve": round(ms_filter, 4)},
            "roofline": r_trace if ms_trace >= ms_shade else r_shade, "roofline_trace": r_trace, "roofline_shade": r_shade,
            "roofline_hbm": {"kernel": "batch filter+resolve pass", "bound": "hbm", "achieved": round(fr_gbs, 1), "peak": hbm_peak,
                             "unit": "GB/s", "frac": round(fr_gbs / hbm_peak, 4) if hbm_peak else None, "traffic": None,
                             "algorithmic_bytes": fr_bytes, "peak_source": hbm_source},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if not args.no_e2e:
            result["e2e"] = batch_e2e(b, torch, views, total_px, args)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_batch_sample(seeds, views, args.cpu_seconds)
        if rank == 0:
            print(json.dumps(result), flush=True)
    finally:
        b.close()


def batch_e2e(b, torch, views, total_px: int, args) -> dict:
    """Per step: every view's camera record from host memory, one batch
    render, every view's Pixels back to pinned host memory."""
    C = np.ascontiguousarray(np.stack([v[3] for v in views]), np.float32)
    host = torch.empty(total_px, dtype=torch.int32).pin_memory()
    stream = torch.cuda.current_stream()
    for _ in range(max(1, args.warmup // 2)):
        b.set_cameras(C)
        b.render()
        b.read_pixels_into(host.data_ptr(), total_px)
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.record(stream)
    for _ in range(args.steps):
        b.set_cameras(C)
        b.render()
        b.read_pixels_into(host.data_ptr(), total_px)
    e.record(stream)
    e.synchronize()
    wall = time.perf_counter() - t0
    ms = a.elapsed_time(e)
    return {"value": round(total_px * args.steps / (ms / 1e3) / 1e6, 3), "unit": UNIT, "h2d_bytes_per_step": int(C.nbytes),
            "d2h_bytes_per_step": total_px * 4, "ms_per_step": round(ms / args.steps, 4),
            "host_wall_ms_per_step": round(wall * 1e3 / args.steps, 4),
            "api": "arbor_batch_set_cameras + arbor_batch_render + arbor_batch_read_pixels (pinned host buffers)"}


def cpu_batch_sample(seeds, views, target_s: float) -> dict:
    """The reference's CPU implementation on evenly strided rows of four of
    the batch's views (one of each resolution where the batch has it)."""
    o, kind = cpu_oracle()
    picked, seen = [], set()
    for v in views:
        if (v[1], v[2]) not in seen:
            seen.add((v[1], v[2]))
            picked.append(v)
    scenes = {}
    rays = 0
    secs = 0.0
    per_view = target_s / len(picked)
    for scene, w, h, C in picked:
        if scene not in scenes:
            scenes[scene] = o.build_scene(seeds[scene])
        bufs = {k: np.zeros(w * h * 4, np.float32) for k in ("Hit", "Linear", "Guide", "Filtered", "History")}
        bufs["Pixels"] = np.zeros(w * h, np.uint32)
        n = min(h, 4 * max(1, o.max_threads()))
        for attempt in range(2):
            rows = np.unique((np.arange(n) * h // n + (h // n) // 2).clip(0, h - 1)).astype(np.int32)
            t0 = time.perf_counter()
            o.frame_rows(scenes[scene], C.copy(), w, h, rows, bufs)
            dt = time.perf_counter() - t0
            if attempt == 0:
                n = int(min(h, max(len(rows), len(rows) * per_view / max(dt, 1e-3))))
        rays += len(rows) * w
        secs += dt
    return {"value": round(rays / secs / 1e6, 4), "unit": UNIT, "cores": o.max_threads(), "kind": kind,
            "sample": f"evenly strided rows of {len(picked)} views of the batch ({', '.join(f'{p[1]}x{p[2]}' for p in picked)}; "
                      f"{rays} primary rays, {secs:.2f} s): trace, shade with sun shadows, filter, resolve",
            "seconds": round(secs, 3)}


def run_reference_batch(args) -> None:
    import workloads

    seeds = workloads.batch_seeds(args.scenes)
    views = workloads.batch_views(args.views, seeds)
    step_s = float(os.environ.get("ARBOR_REFERENCE_STEP_SECONDS", "2.0"))
    samples = [cpu_batch_sample(seeds, views, step_s) for _ in range(args.warmup + args.steps)][args.warmup:]
    value = statistics.mean(x["value"] for x in samples)
    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * statistics.mean(x["seconds"] for x in samples), 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic: procedural scenes grown from the master seeds", "impl": "reference",
            "config": batch_spec(args),
            "cpu_baseline": {k: samples[-1][k] for k in ("unit", "cores", "kind", "sample")} | {"value": round(value, 4)},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- denoiser --
# Multiply-accumulates per pixel of the denoiser network (3x3 convolutions;
# level l runs at 1/4^l of the pixels; the output layer's 3 used channels).
DENOISER_LAYERS = [(16, 32, 0), (32, 32, 0), (32, 64, 1), (64, 64, 1), (64, 96, 2), (96, 96, 2), (96, 128, 3), (128, 128, 3), (224, 96, 2),
                   (96, 96, 2), (160, 64, 1), (64, 64, 1), (96, 32, 0), (32, 32, 0), (32, 3, 0)]
DENOISER_MACS_PER_PIXEL = sum(9 * ci * co / 4 ** lv for ci, co, lv in DENOISER_LAYERS)


def run_denoise(args, rank: int, world: int, local_rank: int) -> None:
    """The learned denoiser at 1920x1080 on a rendered 1-spp forest frame with
    sun shadows: filterLighting, features and the network per frame (weights
    untrained: the time does not depend on their values), against
    filterLighting alone."""
    import ctypes

    import torch
    import torch.distributed as dist

    import arbor_b200 as ab
    import workloads

    W, H = 1920, 1080
    spec = {"workload": "denoise-1080p: learned denoiser (4-level U-Net 32/64/96/128, BF16 tensor cores) on a 1-spp 1920x1080 forest "
                        "frame with sun shadows, per frame: filterLighting + features + network", "width": W, "height": H}
    fr = Frames(ab, {**workload_spec("shadows"), "width": W, "height": H}, torch)
    fr.step(0)
    Nrm = torch.zeros(W * H * 4, device="cuda")
    feat = torch.zeros(W * H * 16, dtype=torch.int16, device="cuda")
    den = torch.zeros(W * H * 4, device="cuda")
    fr.check(ab.call("arbor_shadeGBuffer", fr.P, fr.Nodes, fr.Order, fr.C, fr.Hit, fr.Lin, fr.Gui, Nrm, W, H))
    lib = ab.lib()
    h = ctypes.c_void_p()
    fr.check(lib.arbor_denoiser_create(ctypes.byref(h), 1, W, H, 7, ab.stream_handle()))

    def frame():
        fr.check(ab.call("arbor_filterLighting", fr.Lin, fr.Gui, fr.Hit, fr.Fil, fr.C, W, H))
        fr.check(ab.call("arbor_denoiser_features", fr.Lin, fr.Gui, Nrm, fr.Hit, fr.Fil, W, H, feat))
        fr.check(lib.arbor_denoiser_infer(h, feat.data_ptr(), fr.Fil.data_ptr(), den.data_ptr(), W, H))

    try:
        results = {}
        for backend, name in ((1, "tcgen05"), (0, "mma.sync")):
            fr.check(lib.arbor_denoiser_set_backend(h, backend))
            for _ in range(args.warmup):
                frame()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            sampler = ClockSampler(physical_gpu(local_rank))
            sampler.start()
            time.sleep(0.3)
            launches0 = ab.launches()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(args.steps):
                frame()
            b.record()
            b.synchronize()
            fr.check(lib.arbor_denoiser_check(h))
            results[name] = {"ms": a.elapsed_time(b) / args.steps, "launches": ab.launches() - launches0, "clocks": sampler.stop()}
        ms_filter = time_kernel(torch, lambda: fr.check(ab.call("arbor_filterLighting", fr.Lin, fr.Gui, fr.Hit, fr.Fil, fr.C, W, H)), 20)
    finally:
        lib.arbor_denoiser_destroy(h)
    peaks = measured_peaks()
    peak = peaks.get("bf16_tflops")
    flops = 2.0 * DENOISER_MACS_PER_PIXEL * W * H
    ms = results["tcgen05"]["ms"]
    achieved = flops / (ms / 1e3) / 1e12
    ms_max = max_over_ranks(ms, world)
    line = {
        "metric": METRIC, "value": round(ms_max, 4), "unit": "ms per 1080p frame (denoiser)", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16", "data": "synthetic: rendered forest frame (seed 7, walk frame 0, sun shadows); untrained weights",
        "config": {**spec, "parallelism": f"replicas x{world}",
                   "l2": "per-frame activations (level 0: 96 channels x 2 M pixels x 2 B = 398 MB) exceed the 126 MB L2"},
        "phases_ms": {"denoiser_tcgen05": round(results["tcgen05"]["ms"], 4), "denoiser_mma_sync": round(results["mma.sync"]["ms"], 4),
                      "filterLighting": round(ms_filter, 4)},
        "roofline": {"kernel": "denoiser network (15 convolutions + elementwise), tcgen05", "bound": "tensor", "achieved": round(achieved, 2),
                     "peak": peak, "unit": "TFLOP/s", "frac": round(achieved / peak, 4) if peak else None, "traffic": None,
                     "algorithmic_flops": flops, "macs_per_pixel": round(DENOISER_MACS_PER_PIXEL, 1),
                     "peak_source": ("MEASURED_PEAKS.json bf16_tflops (of measured, burst)" if peaks["source"] == "measured" else "bf16 1590 TFLOP/s (of fallback)")},
        "gpu_launches": int(results["tcgen05"]["launches"]),
        "clocks": results["tcgen05"]["clocks"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main() -> None:
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch

    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local_rank))
    try:
        if args.workload == "batch":
            run_batch(args, rank, world, local_rank)
        elif args.workload == "denoise":
            run_denoise(args, rank, world, local_rank)
        else:
            run_arbor(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
