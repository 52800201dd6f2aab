"""Generate the golden fixtures from the reference's own CPU execution.

    python tests/golden/make_golden.py

Runs the reference harness code built from the reference's sources
(oracle/_ref/libarbor_ref.so, see oracle/Makefile; needs the reference
checkout) and records, for fixed seeds and cameras, SHA-256 digests of every
buffer the render path produces, plus the harness's own recorded check values
(docs/native-checks.log).  The GPU box has no reference checkout, so tests
there compare against these fixtures and against the oracle port.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "arbor-cuda_b200"))
from pyoracle import CAPACITY, OBJECT_COUNT, PS, Oracle  # noqa: E402

import workloads  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")
SEEDS = (0, 1, 7, 42, 1788)
FRAME_W, FRAME_H = 96, 64
TREE_W, TREE_H = 128, 128


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def harness_rays(ref: Oracle, scene: dict) -> list:
    """The harness's 100 BVH rays against exhaustive intersection (tests/native_harness.cpp:82-87)."""
    out = []
    for ray in range(100):
        ro, rd = ref.harness_ray(ray)
        t, oid = ref.trace_tree_ray(scene, ro, rd, 0.0005)
        et, eid = ref.exhaustive_ray(scene["P"], ro, rd, 0.0005)
        out.append({"ro": ro.tolist(), "rd": rd.tolist(), "t": t, "id": oid, "exhaustive_t": et, "exhaustive_id": eid})
    return out


def main() -> None:
    ref = Oracle("reference")
    gold: dict = {"generator": "tests/golden/make_golden.py", "source": "reference harness (tests/native_harness.cpp + Arbor.cu) built by oracle/Makefile"}
    gold["scenes"] = {}
    for seed in SEEDS:
        s = ref.build_scene(seed)
        h = ref.harness_build(seed)
        for k in ("B", "P", "Keys", "Order", "Nodes"):
            assert np.array_equal(s[k], h[k]), (seed, k)
        types = s["P"].reshape(CAPACITY, PS)[:, 3]
        n = s["Nodes"]
        raw = s["RawKeys"]
        gold["scenes"][str(seed)] = {
            **{k: digest(s[k]) for k in ("B", "P", "Keys", "Order", "Nodes", "RawKeys")},
            "root_lo": n[8:11].tolist(), "root_hi": n[12:15].tolist(), "root_count": float(n[11]),
            "wood": int((types == 0).sum()), "leaves": int((types == 1).sum()), "rocks": int((types == 2).sum()),
            "duplicate_keys": int(len(raw[raw != 0xFFFFFFFF]) - len(np.unique(raw[raw != 0xFFFFFFFF]))),
            "order_head": s["Order"][:16].tolist(), "keys_head": s["Keys"][:16].tolist(),
        }
    # bitonic network equals the independent sort (native_harness.cpp:78-80)
    s1 = ref.build_scene(1)
    k, o = s1["RawKeys"].copy(), np.arange(CAPACITY, dtype=np.uint32)
    ref.bitonic(k, o)
    gold["bitonic_equals_sort_seed1"] = bool(np.array_equal(k, s1["Keys"]) and np.array_equal(o, s1["Order"]))

    # Forest frames at seed 1788: every preset, shadows off and on, and the
    # three debug view modes.
    scene = ref.build_scene(1788)
    frames = {}
    cases = [(v, light, 0) for v in workloads.VIEW_PRESETS for light in (0, 1)] + [(2, 0, m) for m in (1, 2, 3)]
    for view, light, mode in cases:
        C = ref.init_camera(scene["P"], 1788)
        I = np.zeros(32, np.float32)
        I[5] = view
        ref.update_camera(C, I, scene["P"], 1.0 / 60, FRAME_W, FRAME_H)
        C[22] = light
        C[15] = mode
        f = ref.frame(scene, C, FRAME_W, FRAME_H)
        frames[f"view{view}_light{light}_mode{mode}"] = {"C": C.tolist(), **{k: digest(v) for k, v in f.items()}}
    gold["frames_1788_96x64"] = frames

    # Single tree, seed 1.
    tree = ref.build_scene(1)
    C = workloads.single_tree_camera(TREE_W, TREE_H)
    f = ref.frame(tree, C, TREE_W, TREE_H, single=True)
    gold["tree_seed1_128"] = {"C": C.tolist(), **{k: digest(v) for k, v in f.items()},
                              "hit_fraction": float(np.mean(f["Hit"][1::4] >= 0))}
    C2 = C.copy()
    C2[22] = 1.0
    f2 = ref.frame(tree, C2, TREE_W, TREE_H, single=True)
    gold["tree_seed1_128_shadows"] = {"C": C2.tolist(), **{k: digest(v) for k, v in f2.items()}}

    # Seeded walk: camera record after each of the first 8 frames.
    walk = []
    Cw = ref.init_camera(scene["P"], 7)
    sc7 = ref.build_scene(7)
    for frame in range(8):
        I, dt = workloads.walk_input(frame)
        ref.update_camera(Cw, I, sc7["P"], dt, 192, 108)
        walk.append(Cw.tolist())
    gold["walk_seed7_C"] = walk
    # The measured walk: camera record after each of the 64 frames at 1920x1080.
    walk = []
    Cw = ref.init_camera(sc7["P"], 7)
    for frame in range(64):
        I, dt = workloads.walk_input(frame)
        ref.update_camera(Cw, I, sc7["P"], dt, 1920, 1080)
        walk.append(Cw.tolist())
    gold["walk_seed7_1080p_C"] = walk

    # The harness's recorded check values.
    rays = harness_rays(ref, scene)
    gold["harness_rays_1788"] = rays
    gold["harness_bvh_max_t_error"] = max(abs(r["t"] - r["exhaustive_t"]) for r in rays if r["t"] < 1e5 and r["exhaustive_t"] < 1e5)
    jump, mono, finite = ref.footprint_sweep(scene["P"], 4)
    gold["footprint_sweep"] = {"max_jump": jump, "monotone": mono, "finite": finite}
    gold["leaf_pairs"] = [list(ref.leaf_pair(scene["P"], k)) for k in range(50)]
    gold["instances_seed7"] = [ref.forest_instance(t, 7).tolist() for t in (0, 1, 17, 100, 161, 162, 323)]
    gold["forest_seeds_seed7"] = [ref.forest_seed(t, 7) for t in range(324)]
    with open(OUT, "w") as fh:
        json.dump(gold, fh, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
