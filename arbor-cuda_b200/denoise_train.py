"""Learned denoiser: training pairs rendered by the tracer, training on the
GPU by the library's own kernels, and evaluation against filterLighting.

    python arbor-cuda_b200/denoise_train.py [--train-views 96] [--eval-views 64]
        [--size 384] [--spp 256] [--steps 1500] [--batch 4] [--lr 5e-4]
        [--warmup 1000] [--hflip] [--loss l1|l2] [--streams 8] [--crop 256]
        [--eval-width 1920 --eval-height 1080] [--eval-spp 64] [--out results.json]

At the stated size (2,048 256x256 pairs' worth of 1/256-spp training pixels,
64 held-out full-HD poses against 256-spp renders; about 35 minutes on one
B200, most of it rendering):

    python arbor-cuda_b200/denoise_train.py --train-views 512 --size 512 --crop 256 \
        --spp 256 --eval-views 64 --eval-width 1920 --eval-height 1080 --eval-spp 256 \
        --steps 40000 --batch 4 --lr 5e-4 --warmup 1000 --hflip --streams 8

Data: views of the 324-tree forest from 16 master seeds at random poses
(1.72 m eye height, sun shadows on), `size` x `size` pixels with the
per-pixel angle of a 1920x1080 frame (C[14] scaled by size / 1080), so a
view is a crop of a full-HD frame.  Sample s of a view renders with
C[9] = s (Halton subpixel jitter and sun-disk jitter per sample, as the
harness's progressive loop sets it, tests/native_harness.cpp:62).  Input: the
1-spp Linear, albedo (Guide), normal (arbor_shadeGBuffer) and depth (Hit);
target: the mean of Linear over `spp` samples.

The network corrects filterLighting's 1-spp output (its base image) using
the features; training minimises L1 (or L2) in log(1 + radiance) with Adam:
each step a batch of random training views (random --crop windows of them
when given), each mirrored with probability
1/2 under --hflip, the learning rate ramped up over --warmup steps and then
decayed on a cosine.  Peak rates of 1e-3 and above diverged on runs of
20,000 steps (loss spikes, then NaN); 5e-4 with the warm-up did not.

Evaluation, on held-out views (other poses; full frames of --eval-width x
--eval-height at C[14] = 0.9 when given, else crops like the training views,
with an --eval-spp target): PSNR against the target
after resolvePixels' tone mapping (exposure, ACES, gamma 1/2.2, vignette;
Arbor.cu:303-304, before quantisation), of
  - filterLighting at 1 spp (Filtered),
  - filterLighting at 4 spp (History after 4 samples: the mean of Filtered),
  - the denoiser at 1 spp,
and frame times at 1920x1080 by CUDA events: trace + shade per sample,
filterLighting, and the denoiser (filterLighting + features + network).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import arbor_b200 as ab  # noqa: E402
import workloads  # noqa: E402


def check(st):
    if st != ab.OK:
        raise RuntimeError(f"{ab.STATUS.get(st)}: {ab.last_error()}")


class Scene:
    def __init__(self, seed: int):
        f = lambda n: torch.zeros(n, dtype=torch.float32, device="cuda")  # noqa: E731
        i = lambda n: torch.zeros(n, dtype=torch.int32, device="cuda")  # noqa: E731
        self.B, self.P, self.Keys, self.Order, self.Nodes = f(2109 * 20), f(32768 * 24), i(32768), i(32768), f(65536 * 8)
        scratch = i(2 * 32768)
        check(ab.call("arbor_buildScene", seed, self.B, self.P, self.Keys, self.Order, self.Nodes, None, scratch))


class Frame:
    """Device images of one view size."""

    def __init__(self, w: int, h: int):
        f = lambda n: torch.zeros(n, dtype=torch.float32, device="cuda")  # noqa: E731
        self.w, self.h = w, h
        n = w * h * 4
        self.Hit, self.Lin, self.Gui, self.Nrm, self.Fil, self.Hist, self.Acc = (f(n) for _ in range(7))
        self.Pix = torch.zeros(w * h, dtype=torch.int32, device="cuda")
        self.feat = torch.zeros(w * h * 16, dtype=torch.int16, device="cuda")
        self.C = f(64)

    def set_view(self, C: np.ndarray) -> None:
        self.C.copy_(torch.from_numpy(C))

    def sample(self, scene: Scene, s: int, gbuffer: bool) -> None:
        """Sample s of the current view: C[9] = s, C[10] = (s == 0) set on the device."""
        check(ab.call("arbor_setSample", self.C, s, int(s == 0)))
        w, h = self.w, self.h
        check(ab.call("arbor_tracePixels", scene.P, scene.Nodes, scene.Order, self.C, self.Hit, w, h))
        if gbuffer:
            check(ab.call("arbor_shadeGBuffer", scene.P, scene.Nodes, scene.Order, self.C, self.Hit, self.Lin, self.Gui, self.Nrm, w, h))
        else:
            check(ab.call("arbor_shadePixels", scene.P, scene.Nodes, scene.Order, self.C, self.Hit, self.Lin, self.Gui, w, h))


def view_states(n: int, seeds: list[int], size: int, seed: int, full: tuple[int, int] | None = None) -> list[tuple[int, np.ndarray]]:
    """n seeded views: size x size crops at the pixel angle of a 1080-row
    frame, or (full = (w, h)) whole frames at the reference's C[14] = 0.9."""
    out = []
    res = ((full[0], full[1]),) if full else ((size, size),)
    for scene, w, h, C in workloads.batch_views(n, seeds, resolutions=res, seed=seed, shadows=True):
        C = C.copy()
        C[14] = np.float32(0.9 if full else 0.9 * size / 1080.0)  # the pixel angle of a 1080-row frame
        out.append((scene, C))
    return out


def render_pair(fr: Frame, scene: Scene, C: np.ndarray, spp: int, eval_baselines: bool) -> dict:
    """1-spp inputs, the spp target and (for evaluation) filterLighting at 1 and 4 spp."""
    n = fr.w * fr.h * 4
    out = {}
    fr.set_view(C)
    for s in range(spp):
        fr.sample(scene, s, gbuffer=(s == 0))
        if s == 0:
            check(ab.call("arbor_filterLighting", fr.Lin, fr.Gui, fr.Hit, fr.Fil, fr.C, fr.w, fr.h))
            check(ab.call("arbor_denoiser_features", fr.Lin, fr.Gui, fr.Nrm, fr.Hit, fr.Fil, fr.w, fr.h, fr.feat))
            out["feat"] = fr.feat.clone()
            out["noisy"] = fr.Lin.clone()
            out["base"] = fr.Fil.clone()
        if eval_baselines and s < 4:
            check(ab.call("arbor_filterResolve", fr.Lin, fr.Gui, fr.Hit, fr.Fil, fr.Hist, fr.Pix, fr.C, fr.w, fr.h))
            if s == 0:
                out["filter1"] = fr.Fil.clone()
            if s == 3:
                out["filter4"] = fr.Hist.clone()
        check(ab.call("arbor_accumulate", fr.Acc, fr.Lin, n, 0.0 if s == 0 else 1.0))
    out["target"] = fr.Acc.clone() / float(spp)
    return out


def render_pairs(frames: list[Frame], jobs: list[tuple[Scene, np.ndarray]], spp: int, eval_baselines: bool) -> list[dict]:
    """render_pair for many views, len(frames) at a time, view k of a group
    on CUDA stream k: a small view's persistent passes leave SMs idle at
    their tails, which the other streams' views fill."""
    streams = [torch.cuda.Stream() for _ in frames]
    out = []
    for g in range(0, len(jobs), len(frames)):
        for k, (scene, C) in enumerate(jobs[g:g + len(frames)]):
            with torch.cuda.stream(streams[k]):
                out.append(render_pair(frames[k], scene, C, spp, eval_baselines))
        torch.cuda.synchronize()
    return out


def tonemap(lin: torch.Tensor, w: int, h: int, exposure: float) -> torch.Tensor:
    """resolvePixels' float colour before quantisation (Arbor.cu:303-304)."""
    c = lin.view(h, w, 4)[..., :3].double() * exposure
    c = ((c * (2.51 * c + 0.03)) / (c * (2.43 * c + 0.59) + 0.14)).clamp(0.0, 1.0)
    c = c.pow(1.0 / 2.2)
    u = (torch.arange(w, device=lin.device, dtype=torch.float64) / w - 0.5) * 2.0
    v = (torch.arange(h, device=lin.device, dtype=torch.float64) / h - 0.5) * 2.0
    vig = 1.0 - 0.09 * (u[None, :] ** 2 + v[:, None] ** 2)
    return (c * vig[..., None]).clamp(0.0, 1.0)


def psnr(a: torch.Tensor, b: torch.Tensor) -> float:
    mse = float(((a - b) ** 2).mean())
    return 10.0 * math.log10(1.0 / max(mse, 1e-12))


def time_ms(fn, reps: int = 10) -> float:
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) / reps


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-views", type=int, default=96)
    ap.add_argument("--eval-views", type=int, default=64)
    ap.add_argument("--size", type=int, default=384)
    ap.add_argument("--spp", type=int, default=256)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=5e-4, help="peak learning rate (cosine decay after --warmup steps of linear ramp)")
    ap.add_argument("--warmup", type=int, default=1000)
    ap.add_argument("--loss", choices=["l1", "l2"], default="l1", help="training loss in log(1 + radiance)")
    ap.add_argument("--scenes", type=int, default=16)
    ap.add_argument("--hflip", action="store_true", help="mirror each training view (horizontal flip) with probability 1/2 per step")
    ap.add_argument("--streams", type=int, default=8, help="training views rendered concurrently, one CUDA stream each")
    ap.add_argument("--crop", type=int, default=0, help="train on random crop x crop windows of the size x size views (default: whole views)")
    ap.add_argument("--eval-width", type=int, default=0, help="evaluate on whole frames of this size (with --eval-height)")
    ap.add_argument("--eval-height", type=int, default=0)
    ap.add_argument("--eval-spp", type=int, default=0, help="samples of the evaluation target (default --spp)")
    ap.add_argument("--out", default="")
    args = ap.parse_args()
    torch.cuda.init()
    lib = ab.lib()
    S = args.size
    seeds = workloads.batch_seeds(args.scenes)
    scenes = {}
    fr = Frame(S, S)
    t0 = time.perf_counter()

    def scene_of(k):
        if k not in scenes:
            scenes[k] = Scene(seeds[k])
        return scenes[k]

    train_views = view_states(args.train_views, seeds, S, seed=11)
    full = (args.eval_width, args.eval_height) if args.eval_width and args.eval_height else None
    EW, EH = full if full else (S, S)
    eval_spp = args.eval_spp or args.spp
    eval_views = view_states(args.eval_views, seeds, S, seed=12, full=full)
    px = S * S
    feats = torch.zeros(args.train_views, px * 16, dtype=torch.int16, device="cuda")
    base = torch.zeros(args.train_views, px * 4, device="cuda")
    target = torch.zeros(args.train_views, px * 4, device="cuda")
    frames = [Frame(S, S) for _ in range(max(1, args.streams))]
    chunk = 64 * len(frames)
    for c0 in range(0, len(train_views), chunk):
        part = train_views[c0:c0 + chunk]
        for j, r in enumerate(render_pairs(frames, [(scene_of(k), C) for k, C in part], args.spp, eval_baselines=False)):
            feats[c0 + j], base[c0 + j], target[c0 + j] = r["feat"], r["base"], r["target"]
    del frames
    efr = Frame(EW, EH) if full else fr
    evals = []
    for k, C in eval_views:
        evals.append(render_pair(efr, scene_of(k), C, eval_spp, eval_baselines=True) | {"C": C})
    n_train = args.train_views
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0

    # training
    h = ctypes.c_void_p()
    R = args.crop if 0 < args.crop <= S else S
    check(lib.arbor_denoiser_create(ctypes.byref(h), args.batch, R, R, 7, None))
    check(lib.arbor_denoiser_set_loss(h, ab.LOSS_L2 if args.loss == "l2" else ab.LOSS_L1))
    rng = np.random.default_rng(1)
    losses = []
    fb = torch.empty(args.batch, R * R * 16, dtype=torch.int16, device="cuda")
    bb = torch.empty(args.batch, R * R * 4, device="cuda")
    tb = torch.empty(args.batch, R * R * 4, device="cuda")
    t0 = time.perf_counter()
    for step in range(args.steps):
        # a batch of random R x R windows of random views, each mirrored with
        # probability 1/2 (--hflip)
        for j in range(args.batch):
            i = int(rng.integers(0, n_train))
            y, x = int(rng.integers(0, S - R + 1)), int(rng.integers(0, S - R + 1))
            flip = bool(args.hflip and rng.integers(0, 2))
            for src, dst, ch in ((feats, fb, 16), (base, bb, 4), (target, tb, 4)):
                v = src[i].view(S, S, ch)[y:y + R, x:x + R]
                dst[j].view(R, R, ch).copy_(v.flip(1) if flip else v)
        lr = 1e-5 + 0.5 * (args.lr - 1e-5) * (1.0 + math.cos(math.pi * step / args.steps))
        if step < args.warmup:
            lr *= (step + 1) / args.warmup
        lv = ctypes.c_float()
        want = step % 50 == 0 or step == args.steps - 1
        check(lib.arbor_denoiser_train_step(h, fb.data_ptr(), bb.data_ptr(), tb.data_ptr(), args.batch, R, R, lr,
                                            ctypes.byref(lv) if want else None))
        if want:
            losses.append((step, round(lv.value, 5)))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0

    # evaluation (views of another size than the training windows: a second
    # denoiser of that size with the trained parameters)
    he = h
    separate = (EW, EH) != (R, R)
    if separate:
        n_par = ctypes.c_size_t()
        check(lib.arbor_denoiser_param_count(h, ctypes.byref(n_par)))
        params = np.zeros(n_par.value, np.float32)
        check(lib.arbor_denoiser_get_params(h, params.ctypes.data, params.size))
        he = ctypes.c_void_p()
        check(lib.arbor_denoiser_create(ctypes.byref(he), 1, EW, EH, 7, None))
        check(lib.arbor_denoiser_set_params(he, params.ctypes.data, params.size))
    den = torch.zeros(EW * EH * 4, device="cuda")
    scores = {"noisy_1spp": [], "filter_1spp": [], "filter_4spp": [], "denoiser_1spp": []}
    for e in evals:
        check(lib.arbor_denoiser_infer(he, e["feat"].data_ptr(), e["base"].data_ptr(), den.data_ptr(), EW, EH))
        exposure = float(e["C"][20])
        ref = tonemap(e["target"], EW, EH, exposure)
        scores["noisy_1spp"].append(psnr(tonemap(e["noisy"], EW, EH, exposure), ref))
        scores["filter_1spp"].append(psnr(tonemap(e["filter1"], EW, EH, exposure), ref))
        scores["filter_4spp"].append(psnr(tonemap(e["filter4"], EW, EH, exposure), ref))
        scores["denoiser_1spp"].append(psnr(tonemap(den, EW, EH, exposure), ref))
    if separate:
        check(lib.arbor_denoiser_destroy(he))
    check(lib.arbor_denoiser_destroy(h))

    # frame times at 1920x1080
    W, H = 1920, 1080
    big = Frame(W, H)
    C = view_states(1, seeds, S, seed=12)[0][1].copy()
    C[14] = np.float32(0.9)
    C[32], C[33] = W, H
    sc = scene_of(view_states(1, seeds, S, seed=12)[0][0])
    big.set_view(C)
    big.sample(sc, 0, gbuffer=True)
    ms_sample = time_ms(lambda: big.sample(sc, 1, gbuffer=False), 5)
    ms_filter = time_ms(lambda: check(ab.call("arbor_filterLighting", big.Lin, big.Gui, big.Hit, big.Fil, big.C, W, H)))
    hd = ctypes.c_void_p()
    check(lib.arbor_denoiser_create(ctypes.byref(hd), 1, W, H, 7, None))
    bigden = torch.zeros(W * H * 4, device="cuda")

    def run_denoiser():
        check(ab.call("arbor_filterLighting", big.Lin, big.Gui, big.Hit, big.Fil, big.C, W, H))
        check(ab.call("arbor_denoiser_features", big.Lin, big.Gui, big.Nrm, big.Hit, big.Fil, W, H, big.feat))
        check(lib.arbor_denoiser_infer(hd, big.feat.data_ptr(), big.Fil.data_ptr(), bigden.data_ptr(), W, H))

    ms_denoiser = time_ms(run_denoiser)
    check(lib.arbor_denoiser_destroy(hd))
    mean = {k: round(float(np.mean(v)), 3) for k, v in scores.items()}
    result = {
        "denoiser": "4-level U-Net 32/64/96/128, 3x3, BF16 weights and activations, FP32 accumulation; forward "
                    "convolutions and most of the backward data pass on tcgen05 (TMEM accumulators), weight gradients on "
                    "mma.sync m16n8k16 folded in a fixed order",
        "data": {"train_views": args.train_views, "eval_views": args.eval_views, "size": S, "spp_target": args.spp, "scenes": args.scenes, "hflip": bool(args.hflip), "streams": args.streams, "crop": R,
                 "eval_size": [EW, EH], "eval_spp_target": eval_spp, "render_seconds": round(t_data, 1)},
        "train": {"steps": args.steps, "batch": args.batch, "lr": args.lr, "warmup": args.warmup, "loss_kind": args.loss, "seconds": round(t_train, 2),
                  "ms_per_step": round(1e3 * t_train / max(1, args.steps), 3), "loss": losses},
        "psnr_db_mean": mean,
        "psnr_db_min": {k: round(float(np.min(v)), 3) for k, v in scores.items()},
        "gap_denoiser_vs_filter4_db": round(mean["denoiser_1spp"] - mean["filter_4spp"], 3),
        "ms_1080p": {"trace_shade_per_sample_shadows": round(ms_sample, 3), "filterLighting": round(ms_filter, 4),
                     "denoiser_filter_features_network": round(ms_denoiser, 3),
                     "frame_1spp_denoiser": round(ms_sample + ms_denoiser, 3),
                     "frame_4spp_filter": round(4 * ms_sample + 4 * ms_filter, 3)},
    }
    line = json.dumps(result)
    print(line, flush=True)
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(line + "\n")


if __name__ == "__main__":
    main()
