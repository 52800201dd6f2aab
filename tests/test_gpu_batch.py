"""The batched multi-view renderer on the GPU.

Each view of a batch must render as the single-image entries render it
(arbor_tracePixels, arbor_shadePixels, arbor_filterResolve on the same scene
buffers and camera record):
  - bit-identical for configurations whose warps cover the same pixels as
    the single-image kernels (16x16 tiles, queue depth 16), whatever the CTAs
    per SM and the tile order;
  - for the other tile shapes and queue depths, hit IDs agree on >= 99.99%
    of pixels: the warp batch then groups different rays, which changes only
    the order in which exactly equal hit distances are met.
One view is also checked against the CPU oracle with the render tests' bars.
The benchmark's own batch (64 views of 16 forests at four resolutions) is
held to the same rules: every view bit-identical to the single-image entries,
and one view of each resolution against the oracle on a band of rows.
"""
import ctypes

import numpy as np
import pytest

import arbor_b200 as ab
import workloads
from conftest import u32
from gpu_util import dev_array

pytestmark = pytest.mark.gpu

SIZES = ((96, 64), (160, 90), (64, 48), (200, 120), (33, 17), (128, 72))
SEEDS = [7, 1788]
IMAGES = ("Hit", "Linear", "Guide", "Filtered", "History")


def make_views(shadows=True):
    views = []
    for v, (w, h) in enumerate(SIZES):
        scene = v % len(SEEDS)
        r = [workloads.rnd(50 + 4 * v + k, 11) for k in range(4)]
        C = workloads.view_pose_state(SEEDS[scene], w, h, (r[0] * 2 - 1) * 120.0, (r[1] * 2 - 1) * 120.0, r[2] * 6.2831853,
                                      -0.05 + 0.25 * r[3], shadows=shadows and v % 3 != 2)
        views.append((scene, w, h, C))
    return views


class Batch:
    def __init__(self, views, seeds=SEEDS):
        self.lib = ab.lib()
        self.views = views
        arr = (ab.BatchView * len(views))()
        for i, (scene, w, h, C) in enumerate(views):
            arr[i].scene, arr[i].width, arr[i].height = scene, w, h
            arr[i].C[:] = [float(x) for x in C]
        sd = (ctypes.c_int * len(seeds))(*seeds)
        self.h = ctypes.c_void_p()
        st = self.lib.arbor_batch_create(ctypes.byref(self.h), sd, len(seeds), arr, len(views), None)
        assert st == ab.OK, ab.last_error()

    def call(self, name, *args):
        st = getattr(self.lib, name)(self.h, *args)
        assert st == ab.OK, f"{name}: {ab.last_error()}"

    def buffers(self, v) -> ab.EngineBuffers:
        b = ab.EngineBuffers()
        self.call("arbor_batch_view_buffers", v, ctypes.byref(b))
        return b

    def images(self, v) -> dict:
        _, w, h, _ = self.views[v]
        b = self.buffers(v)
        out = {k: dev_array(getattr(b, k), w * h * 4) for k in IMAGES}
        out["Pixels"] = dev_array(b.Pixels, w * h, np.uint32)
        return out

    def configure(self, tile_width, ctas, order, queue):
        self.call("arbor_batch_configure", ctypes.byref(ab.BatchConfig(tile_width, ctas, order, queue)))

    def close(self):
        self.lib.arbor_batch_destroy(self.h)


def single_image_device(cuda, gu, batch, v) -> dict:
    """The view rendered by the single-image entries on the batch's own scene
    buffers, left on the device."""
    _, w, h, C = batch.views[v]
    b = batch.buffers(v)
    dC = gu.dev(C)
    bufs = gu.render_buffers(w, h)
    gu.ok(cuda.call("arbor_tracePixels", b.P, b.Nodes, b.Order, dC, bufs["Hit"], w, h))
    gu.ok(cuda.call("arbor_shadePixels", b.P, b.Nodes, b.Order, dC, bufs["Hit"], bufs["Linear"], bufs["Guide"], w, h))
    gu.ok(cuda.call("arbor_filterResolve", bufs["Linear"], bufs["Guide"], bufs["Hit"], bufs["Filtered"], bufs["History"], bufs["Pixels"],
                    dC, w, h))
    return bufs


def single_image(cuda, gu, batch, v):
    """The view rendered by the single-image entries, copied to the host."""
    bufs = single_image_device(cuda, gu, batch, v)
    return {k: gu.host(t, np.uint32 if k == "Pixels" else None) for k, t in bufs.items()}


@pytest.fixture(scope="module")
def gu():
    import gpu_util

    return gpu_util


@pytest.fixture(scope="module")
def batch(cuda):
    b = Batch(make_views())
    yield b
    b.close()


@pytest.fixture(scope="module")
def singles(cuda, gu, batch):
    return [single_image(cuda, gu, batch, v) for v in range(len(batch.views))]


@pytest.mark.parametrize("ctas,order", [(2, 0), (1, 1)])
def test_batch_equals_single_image_entries(cuda, gu, batch, singles, ctas, order):
    batch.configure(16, ctas, order, 16)
    batch.call("arbor_batch_render")
    for v in range(len(batch.views)):
        got = batch.images(v)
        for k in IMAGES + ("Pixels",):
            assert np.array_equal(u32(got[k]), u32(singles[v][k])), f"view {v} {k}"


@pytest.mark.parametrize("tw,queue", [(32, 16), (16, 12), (32, 12)])
def test_batch_other_tilings_agree(cuda, gu, batch, singles, tw, queue):
    batch.configure(tw, 2, 0, queue)
    batch.call("arbor_batch_render")
    differ = total = 0
    for v in range(len(batch.views)):
        got, want = batch.images(v), singles[v]
        g, r = got["Hit"].reshape(-1, 4), want["Hit"].reshape(-1, 4)
        differ += int(np.count_nonzero((g[:, 1] != r[:, 1]) | (g[:, 2] != r[:, 2])))
        total += len(g)
    print(f"[batch tile {tw} queue {queue}] {differ} of {total} pixels differ in hit ids")
    assert differ <= max(1, total // 10000)


def test_batch_view_against_oracle(cuda, gu, oracle, scenes, batch):
    batch.configure(16, 2, 0, 16)
    batch.call("arbor_batch_render")
    v = 3  # 200 x 120, seed 1788, shadows on
    scene, w, h, C = batch.views[v]
    ref = oracle.frame(scenes(SEEDS[scene]), C.copy(), w, h)
    got = batch.images(v)
    g, r = got["Hit"].reshape(-1, 4), ref["Hit"].reshape(-1, 4)
    agree = float(np.mean((g[:, 1] == r[:, 1]) & (g[:, 2] == r[:, 2])))
    err = np.max(np.abs(got["Linear"].reshape(-1, 4)[:, :3] - ref["Linear"].reshape(-1, 4)[:, :3])
                 / np.maximum(1.0, np.abs(ref["Linear"].reshape(-1, 4)[:, :3])), 1)
    print(f"[batch view {v} vs oracle] id agreement {agree:.5f}; radiance within 2e-3 on {np.mean(err <= 2e-3):.5f}")
    assert agree >= 0.999
    assert np.mean(err <= 2e-3) >= 0.995


def test_batch_set_cameras_and_pixels(cuda, gu, batch, singles):
    """New cameras through arbor_batch_set_cameras render as the single-image
    path renders them; arbor_batch_read_pixels returns every view's Pixels
    back to back."""
    batch.configure(16, 2, 0, 16)
    moved = []
    for scene, w, h, C in batch.views:
        C2 = C.copy()
        C2[0] += 1.5
        C2[4] += 1.5
        moved.append((scene, w, h, C2))
    flat = np.ascontiguousarray(np.stack([m[3] for m in moved]), np.float32)
    batch.call("arbor_batch_set_cameras", flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(moved))
    batch.call("arbor_batch_render")
    info = ab.BatchInfo()
    batch.call("arbor_batch_inspect", ctypes.byref(info))
    assert info.n_views == len(SIZES) and info.n_scenes == len(SEEDS) and info.launches_per_render == 5
    assert info.total_pixels == sum(w * h for w, h in SIZES)
    px = np.zeros(info.total_pixels, np.uint32)
    batch.call("arbor_batch_read_pixels", px.ctypes.data_as(ctypes.c_void_p), px.size)
    saved = batch.views
    batch.views = moved
    try:
        off = 0
        for v, (_, w, h, _) in enumerate(moved):
            want = single_image(cuda, gu, batch, v)
            assert np.array_equal(px[off:off + w * h], want["Pixels"]), f"view {v}"
            off += w * h
    finally:
        batch.views = saved
        flat = np.ascontiguousarray(np.stack([m[3] for m in saved]), np.float32)
        batch.call("arbor_batch_set_cameras", flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(saved))


def test_batch_autotune(cuda, gu, batch, singles):
    best = ab.BatchConfig()
    ms = (ctypes.c_float * 16)()
    batch.call("arbor_batch_autotune", 3, ctypes.byref(best), ms)
    times = list(ms)
    print("[batch autotune] ms:", [round(t, 3) for t in times], "->", best.as_dict())
    assert all(t > 0 for t in times)
    assert best.tile_width in (16, 32) and best.ctas_per_sm in (1, 2) and best.order in (0, 1) and best.queue in (12, 16)
    k = (best.tile_width == 32) * 8 + (best.ctas_per_sm == 2) * 4 + best.order * 2 + (best.queue == 16)
    assert times[k] == min(times)
    cur = ab.BatchConfig()
    batch.call("arbor_batch_get_config", ctypes.byref(cur))
    assert cur.as_dict() == best.as_dict()
    batch.call("arbor_batch_render")
    differ = total = 0
    for v in range(len(batch.views)):
        g, r = batch.images(v)["Hit"].reshape(-1, 4), singles[v]["Hit"].reshape(-1, 4)
        differ += int(np.count_nonzero(g[:, 1] != r[:, 1]))
        total += len(g)
    assert differ <= max(1, total // 10000)


def test_batch_rejections(cuda):
    lib = ab.lib()
    h = ctypes.c_void_p()
    one = (ab.BatchView * 1)()
    one[0].scene, one[0].width, one[0].height = 0, 64, 64
    one[0].C[:] = [float(x) for x in workloads.view_pose_state(7, 64, 64, 0.0, 0.0, 0.0, 0.0)]
    seeds = (ctypes.c_int * 1)(7)
    assert lib.arbor_batch_create(ctypes.byref(h), seeds, 1, one, 1, None) == ab.OK
    bad = ab.BatchConfig(24, 2, 0, 8)
    assert lib.arbor_batch_configure(h, ctypes.byref(bad)) == ab.ERR_VALUE
    assert lib.arbor_batch_view_buffers(h, 1, ctypes.byref(ab.EngineBuffers())) == ab.ERR_VALUE
    px = np.zeros(10, np.uint32)
    assert lib.arbor_batch_read_pixels(h, px.ctypes.data_as(ctypes.c_void_p), px.size) == ab.ERR_LIMIT
    assert lib.arbor_batch_destroy(h) == ab.OK


# ------------------------------------------------- the 64-view benchmark batch --
# The benchmark's batch: 64 seeded views of 16 resident forests (master seed 7
# and 15 drawn from it) at 320x180, 640x360, 1280x720 and 1920x1080, sun
# shadows on, as workloads.batch_views lays them out.
BIG_VIEWS = 64
BIG_SCENES = 16


@pytest.fixture(scope="module")
def batch64(cuda):
    seeds = workloads.batch_seeds(BIG_SCENES)
    b = Batch(workloads.batch_views(BIG_VIEWS, seeds), seeds)
    b.seeds = seeds
    yield b
    b.close()


def test_batch_64_views_equal_single_image_entries(cuda, gu, batch64):
    """Every view of the 64-view mixed-resolution batch, rendered in one graph
    launch, is bit-identical in Hit, Linear, Guide, Filtered, History and
    Pixels to the single-image entries on the same scene buffers."""
    import torch

    batch64.configure(16, 2, 0, 16)
    batch64.call("arbor_batch_render")
    pixels = 0
    for v in range(len(batch64.views)):
        _, w, h, _ = batch64.views[v]
        b = batch64.buffers(v)
        want = single_image_device(cuda, gu, batch64, v)
        for k in IMAGES + ("Pixels",):
            n = w * h * (1 if k == "Pixels" else 4)
            assert torch.equal(gu.dev_bits(getattr(b, k), n), want[k].view(torch.int32)), f"view {v} ({w}x{h}) {k}"
        pixels += w * h
        del want
    print(f"[batch 64 views] {pixels} pixels bit-identical to the single-image entries")
    assert pixels == sum(w * h for _, w, h, _ in batch64.views)


def first_view_of_each_size(views) -> list[int]:
    first = {}
    for v, (_, w, h, _) in enumerate(views):
        first.setdefault((w, h), v)
    return sorted(first.values())


def test_batch_64_view_bands_against_oracle(cuda, gu, oracle, scenes, batch64):
    """One view of each resolution of the 64-view batch against the oracle on
    a band of 24 rows through the image centre: trace and shade on the band,
    filter and resolve on its 20 interior rows (the filter reads 2 rows either
    side).  Bars: IDs on >= 99.9 % of band pixels, Linear within 2e-3 on
    >= 99.5 %, Filtered within 2e-3 and Pixels within one byte on >= 99 % of
    interior pixels."""
    batch64.configure(16, 2, 0, 16)
    batch64.call("arbor_batch_render")
    for v in first_view_of_each_size(batch64.views):
        scene, w, h, C = batch64.views[v]
        y0, y1 = h // 2 - 12, h // 2 + 12
        sc = scenes(batch64.seeds[scene])
        Hit = oracle.trace(sc, C.copy(), w, h, y0, y1)
        Linear, Guide = oracle.shade(sc, C.copy(), Hit, w, h, y0, y1)
        Filtered = oracle.filter(Linear, Guide, Hit, C.copy(), w, h, y0 + 2, y1 - 2)
        Pixels = oracle.resolve(Filtered, np.zeros(w * h * 4, np.float32), C.copy(), w, h, y0 + 2, y1 - 2)
        got = batch64.images(v)
        band, inner = slice(y0 * w, y1 * w), slice((y0 + 2) * w, (y1 - 2) * w)
        g, r = got["Hit"].reshape(-1, 4)[band], Hit.reshape(-1, 4)[band]
        agree = float(np.mean((g[:, 1] == r[:, 1]) & (g[:, 2] == r[:, 2])))
        errL = gu.rel_err(got["Linear"].reshape(-1, 4)[band, :3], Linear.reshape(-1, 4)[band, :3]).max(1)
        errF = gu.rel_err(got["Filtered"].reshape(-1, 4)[inner, :3], Filtered.reshape(-1, 4)[inner, :3]).max(1)
        pg = got["Pixels"][inner].view(np.uint8).reshape(-1, 4).astype(int)
        pr = Pixels.view(np.uint8).reshape(-1, 4)[inner].astype(int)
        bytes_ok = float(np.mean(np.abs(pg - pr).max(1) <= 1))
        print(f"[batch 64 view {v}: {w}x{h}, scene seed {batch64.seeds[scene]}] id agreement {agree:.5f}; "
              f"Linear within 2e-3 {np.mean(errL <= 2e-3):.5f}; Filtered {np.mean(errF <= 2e-3):.5f}; Pixels {bytes_ok:.5f}")
        assert np.mean(r[:, 1] >= 0) > 0.05, f"view {v}: the band should hit trees"
        assert agree >= 0.999
        assert np.mean(errL <= 2e-3) >= 0.995
        assert np.mean(errF <= 2e-3) >= 0.99
        assert bytes_ok >= 0.99


def test_batch_64_views_hit_ids_against_oracle(cuda, gu, oracle, scenes, batch64):
    """Every view of the 64-view batch against the oracle's trace on 8 rows
    through its centre: hit IDs agree on >= 99.9 % of all these pixels and
    on >= 99.5 % of each view's (a view's 8 rows hold 2,560 to 15,360
    pixels, so a handful of silhouette pixels is a per-mille)."""
    batch64.configure(16, 2, 0, 16)
    batch64.call("arbor_batch_render")
    differ = total = 0
    worst = (1.0, -1)
    for v, (scene, w, h, C) in enumerate(batch64.views):
        y0, y1 = h // 2 - 4, h // 2 + 4
        ref = oracle.trace(scenes(batch64.seeds[scene]), C.copy(), w, h, y0, y1).reshape(-1, 4)[y0 * w:y1 * w]
        got = dev_array(batch64.buffers(v).Hit + y0 * w * 16, (y1 - y0) * w * 4).reshape(-1, 4)
        d = int(np.count_nonzero((got[:, 1] != ref[:, 1]) | (got[:, 2] != ref[:, 2])))
        differ += d
        total += len(ref)
        worst = min(worst, (1.0 - d / len(ref), v))
    print(f"[batch 64 views vs oracle, 8 rows each] {differ} of {total} pixels differ in hit IDs; worst view {worst[1]} at {worst[0]:.5f}")
    assert 1.0 - differ / total >= 0.999
    assert worst[0] >= 0.995
