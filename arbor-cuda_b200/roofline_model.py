"""Algorithmic work of one tracePixels launch, for the FP32 roofline.

The trace kernel is bound by FP32 issue, not HBM: its 5.7 MB scene stays in
L2.  Its algorithmic work is counted, not estimated from the clock: a
counting build of the same traversal/intersection code (count.cu,
arbor_traceWork) tallies, for the measured frame, how often each work event
happens; each event is weighted by the FP32 operations the reference's
source performs for it (Arbor.cu line cited per weight), counting every
add, subtract, multiply, divide, square root, min, max, abs, floor and each
call of a transcendental function (sin, cos, exp, pow, atan2) as one
operation.  Integer hashing, conversions and comparisons are not counted.

Peak: the arithmetic is compiled without FMA contraction (the reference's
rounding), so the usable FP32 rate is one operation per lane per cycle:
148 SMs x 128 lanes x the SM clock measured during the run.
"""
from __future__ import annotations

import numpy as np

# FP32 operations per event (see the module docstring for what counts).
WEIGHTS = {
    # cameraRay + ground plane + world-box clip + DDA setup (Arbor.cu:51, 239-244, 252)
    "ray": 100,
    # one DDA cell: bounding-sphere test + next-crossing update (Arbor.cu:186, 246-248)
    "cell": 22,
    # tree entry: local point/direction transforms, inverse direction, scale of cone/best (Arbor.cu:67-68, 247)
    "tree": 40,
    # one node box test: slab test + acceptance (Arbor.cu:38, 223-224)
    "node": 23,
    # primary wood test: bark frame, tapered tube with caps, bounds, slab, eps, band weights (Arbor.cu:148, 188-198)
    "wood": 254,
    # one SDF march step: point, woodField without the bark body, step update (Arbor.cu:170, 199)
    "march": 60,
    # bark relief past the early-out: woodUV, Voronoi 3x3, two noise3 (Arbor.cu:148-169)
    "bark": 371,
    # shadow wood: mean radii + tube (Arbor.cu:193)
    "wood_shadow": 138,
    # leaf test: wind-rotated frame, projections, petiole tube, box clip (Arbor.cu:171-172, 203-206)
    "leaf": 233,
    # leaf reaching Newton: start value, band weights, final residual and outline test (Arbor.cu:209, 215-216)
    "newton_start": 79,
    # one Newton iteration: five height-field evaluations and the update (Arbor.cu:174, 210-214)
    "newton": 140,
    # stone ellipsoid (Arbor.cu:219)
    "stone": 32,
    # shadow segment: world-box clip and DDA setup of traceForest, transmission and origin update (Arbor.cu:239-244, 272)
    "segment": 70,
}
EVENTS = ["ray", "cell", "tree", "node", "wood", "march", "bark", "wood_shadow", "leaf", "newton_start", "newton", "stone", "segment"]


def count_events(ab, P, Nodes, Order, C, width: int, height: int, single_tree: bool, torch, Hit=None) -> dict:
    """Event totals of one tracePixels launch, or of one shadePixels launch
    on the Hit records `Hit` when given."""
    n = int(ab.lib().arbor_trace_work_slots(width, height))
    slots = torch.zeros(n, dtype=torch.int32, device="cuda")
    if Hit is None:
        st = ab.call("arbor_traceWork", P, Nodes, Order, C, width, height, int(single_tree), slots)
    else:
        st = ab.call("arbor_shadeWork", P, Nodes, Order, C, Hit, width, height, int(single_tree), slots)
    if st != ab.OK:
        raise RuntimeError(ab.last_error())
    per = slots.view(-1, 16).to(torch.int64).sum(0).cpu().numpy()
    return {name: int(per[i]) for i, name in enumerate(EVENTS)}


def add_counts(a: dict, b: dict) -> dict:
    return {k: a.get(k, 0) + b.get(k, 0) for k in EVENTS}


def flops(counts: dict) -> int:
    return int(sum(WEIGHTS[k] * counts[k] for k in EVENTS))


# DRAM traffic per unit, measured with ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) on one 960x544 launch of the forest walk's first
# frame (seed 7, cold caches): the trace kernel moved 5.33 MB for 522,240
# primary rays, the shadow pass of shadePixels 20.31 MB for 522,240 pixels
# (warp-batch queue depth 12).
# The 5.7 MB scene stays in L2, so the traffic grows with the pixel count;
# bench lines scale these to their launch.
TRACE_DRAM_BYTES_PER_RAY = 10.2
SHADOW_DRAM_BYTES_PER_PIXEL = 38.9
TRAFFIC_SOURCE = "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 960x544 forest launch, scaled by units to this launch"


def roofline_entry(kernel: str, counts: dict, pixels: int, ms: float, fp32_peak_tops: float, sm_clock_mhz: float,
                   traffic: int | None = None, traffic_source: str | None = None) -> dict:
    """FP32 roofline line of one launch whose counted events are `counts`
    over `pixels` pixels, timed at `ms` per launch; `traffic` is the
    launch's DRAM bytes where a capture of the kernel exists."""
    ops = flops(counts)
    achieved = ops / (ms / 1e3) / 1e12
    pixels = max(1, pixels)
    return {
        "kernel": kernel, "bound": "fp32", "achieved": round(achieved, 3), "peak": round(fp32_peak_tops, 2),
        "unit": "TFLOP/s", "frac": round(achieved / fp32_peak_tops, 4), "traffic": traffic,
        **({"traffic_source": traffic_source} if traffic is not None else {}),
        "algorithmic_flops": ops, "flops_per_pixel": round(ops / pixels, 1),
        "events_per_pixel": {k: round(v / pixels, 3) for k, v in counts.items() if v},
        "peak_source": f"derived: 148 SM x 128 FP32 lanes x {sm_clock_mhz:.0f} MHz measured SM clock, one non-fused op per lane per "
                       "cycle (no FP32 peak in MEASURED_PEAKS.json)",
        "ms_per_launch": round(ms, 4),
    }


def trace_roofline(ab, fr, torch, ms_trace: float, fp32_peak_tops: float, sm_clock_mhz: float) -> dict:
    counts = count_events(ab, fr.P, fr.Nodes, fr.Order, fr.C, fr.w, fr.h, fr.spec["single_tree"], torch)
    traffic = None if fr.spec["single_tree"] else int(TRACE_DRAM_BYTES_PER_RAY * fr.w * fr.h)
    return roofline_entry("tracePixels", counts, fr.w * fr.h, ms_trace, fp32_peak_tops, sm_clock_mhz, traffic,
                          TRAFFIC_SOURCE + " (trace_pool_kernel)")


def shade_roofline(ab, fr, torch, ms_shade: float, fp32_peak_tops: float, sm_clock_mhz: float) -> dict:
    counts = count_events(ab, fr.P, fr.Nodes, fr.Order, fr.C, fr.w, fr.h, fr.spec["single_tree"], torch, Hit=fr.Hit)
    shadows = bool(fr.spec.get("shadows")) and not fr.spec["single_tree"]
    traffic = int(SHADOW_DRAM_BYTES_PER_PIXEL * fr.w * fr.h) if shadows else None
    return roofline_entry("shadePixels", counts, fr.w * fr.h, ms_shade, fp32_peak_tops, sm_clock_mhz, traffic,
                          TRAFFIC_SOURCE + " (shadow_pool_kernel; the compose pass, 64 B/px, is not included)")
