"""The C++ engine (src/engine.js restated) on the GPU: the host contract the
reference tests with a fake device (tests/source.test.mjs:6) and the real-GPU
checks of tests/browser.js:5-13."""
import zlib

import numpy as np
import pytest
import torch

import arbor_b200 as ab
from gpu_util import dev_array

pytestmark = pytest.mark.gpu


def fingerprint(a: np.ndarray) -> int:
    return zlib.crc32(a.tobytes())


@pytest.fixture()
def engine(cuda):
    e = ab.Engine(512, 320, seed=1788)
    yield e
    e.close()


def test_create_rounds_size_and_builds_scene(engine):
    info = engine.inspect()
    assert (info.width, info.height, info.seed) == (512, 320, 1788)
    assert info.scene_bytes == 5673744 and info.scene_bytes < 7 * 1048576
    b = engine.buffers()
    P = dev_array(b.P, 32768 * 24)
    types = P.reshape(-1, 24)[:, 3]
    assert (types == 0).sum() == 5124 and (types == 1).sum() == 24192
    nodes = dev_array(b.Nodes, 16)
    assert nodes[11] == 29412
    keys = dev_array(b.Keys, 32768, np.uint32)
    assert (np.diff(keys.astype(np.int64)) >= 0).all(), "GPU sort result is sorted"
    assert np.isfinite(P).all()


def test_frame_contract(engine):
    b = engine.buffers()
    before = fingerprint(dev_array(b.P, 32768 * 24))
    engine.set_input([0] * 5 + [2] + [0] * 26)  # view preset 2
    n0 = ab.launches()
    engine.frame(1 / 60)
    torch.cuda.synchronize()
    assert ab.launches() - n0 == engine.inspect().launches_per_frame == 6
    engine.set_input([0] * 32)
    engine.frame(1 / 60)
    px = np.empty(512 * 320, np.uint32)
    engine.read_pixels_into(px.ctypes.data, px.size)
    assert ((px >> 24) == 255).all(), "opaque alpha"
    r = px & 255
    assert int(r.max()) - int(r.min()) > 40, "non-constant frame"
    lin = dev_array(b.Linear, 512 * 320 * 4)
    assert np.isfinite(lin).all() and (lin >= 0).all()
    assert fingerprint(dev_array(b.P, 32768 * 24)) == before, "camera never touches geometry"
    cam = np.array(engine.inspect().camera)
    assert cam[3] < 2 and cam[24] == 2  # preset executed; two frames counted


def test_resize_generate_and_errors(engine):
    engine.resize(700, 470)
    info = engine.inspect()
    assert (info.width, info.height) == (704, 472)
    engine.frame(1 / 60)
    engine.generate(42)
    assert engine.inspect().seed == 42
    with pytest.raises(ab.ArborError) as ei:
        engine.generate(-1)
    assert ei.value.status == ab.ERR_VALUE
    with pytest.raises(ab.ArborError):
        engine.generate(1000001)
    with pytest.raises(ab.ArborError) as ei:
        engine.resize(100000, 100000)
    assert ei.value.status == ab.ERR_LIMIT
    with pytest.raises(ab.ArborError):
        engine.frame(float("nan"))
    engine.dispose()
    with pytest.raises(ab.ArborError) as ei:
        engine.frame(1 / 60)
    assert ei.value.status == ab.ERR_STATE


def test_small_resolution_rounds_up(cuda):
    e = ab.Engine(10, 10, seed=3)
    info = e.inspect()
    assert (info.width, info.height) == (320, 192)
    e.frame(0.0)
    e.close()


def test_single_tree_engine(cuda):
    e = ab.Engine(320, 192, seed=1, single_tree=True)
    e.frame(1 / 60)
    b = e.buffers()
    hit = dev_array(b.Hit, 320 * 192 * 4).reshape(-1, 4)
    assert (hit[:, 2] == -1).all()
    e.close()


def test_timing_reports_phases(engine):
    engine.set_timing(True)
    engine.frame(1 / 60)
    info = engine.inspect()
    assert info.ms_visibility > 0 and info.ms_lighting > 0 and info.ms_resolve > 0


def test_save_ppm_matches_pixels(cuda, tmp_path):
    """arbor_engine_save_ppm writes the frame the engine holds, in the
    harness's PPM format (tests/native_harness.cpp:53)."""
    e = ab.Engine(320, 192, seed=1788)
    try:
        e.frame(1 / 60)
        info = e.inspect()
        px = np.zeros(info.width * info.height, np.uint32)
        e.read_pixels_into(px.ctypes.data, px.size)
        path = tmp_path / "frame.ppm"
        ab.check(ab.lib().arbor_engine_save_ppm(e.handle, str(path).encode()))
        rgb = np.stack([px & 255, (px >> 8) & 255, (px >> 16) & 255], 1).astype(np.uint8).tobytes()
        assert path.read_bytes() == f"P6\n{info.width} {info.height}\n255\n".encode() + rgb
    finally:
        e.close()
