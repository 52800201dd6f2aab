"""The C-ABI library without a GPU: it loads, exports every symbol the header
declares, and rejects bad arguments before touching the device (the checks
of vendor/cuda-webshader/runtime/runtime.js:18-22, 323-325, 352).

Every call here fails validation, so no kernel is launched; the fake device
addresses are never dereferenced.
"""
import ctypes
import os
import re

import pytest

import arbor_b200 as ab

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "arbor.h")
A = 0x10000000  # fake, 256-byte aligned device addresses (never dereferenced)
MB = 1 << 20


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(arbor_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    return ab.lib()


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 12 + 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(ab.SIGNATURES), set(names) ^ set(ab.SIGNATURES)


def test_the_twelve_reference_entries_are_declared():
    names = declared_functions()
    for entry in ("growTree", "makePrimitives", "makeKeys", "sortPass", "makeBounds", "reduceBounds", "initCamera",
                  "updateCamera", "tracePixels", "shadePixels", "filterLighting", "resolvePixels"):
        assert f"arbor_{entry}" in names


def test_status_names(lib):
    assert lib.arbor_status_name(0) == b"ARBOR_OK"
    assert lib.arbor_status_name(4) == b"ARBOR_ERR_ALIAS"
    assert lib.arbor_status_name(99) == b"ARBOR_ERR_UNKNOWN"
    assert lib.arbor_sort_scratch_bytes() == 2 * 32768 * 4


def test_null_buffers_rejected(lib):
    assert lib.arbor_tracePixels(None, A, A + 4 * MB, A + 8 * MB, A + 16 * MB, 64, 64, None) == ab.ERR_NULL
    assert b"P" in lib.arbor_last_error()
    assert lib.arbor_growTree(None, 0, 1, None) == ab.ERR_NULL
    assert lib.arbor_makeKeys(A, None, A + 8 * MB, None) == ab.ERR_NULL


def test_misaligned_buffers_rejected(lib):
    assert lib.arbor_tracePixels(A + 4, A + 4 * MB, A + 8 * MB, A + 9 * MB, A + 16 * MB, 64, 64, None) == ab.ERR_ALIGN
    assert lib.arbor_makePrimitives(A + 2, A + 4 * MB, 1, None) == ab.ERR_ALIGN


def test_writable_aliasing_rejected(lib):
    # Hit overlapping P (runtime.js:325)
    assert lib.arbor_tracePixels(A, A + 4 * MB, A + 8 * MB, A + 9 * MB, A + 64, 64, 64, None) == ab.ERR_ALIAS
    assert b"aliasing" in lib.arbor_last_error()
    # Keys and Order the same buffer
    assert lib.arbor_sortPass(A, A, 1, 2, None) == ab.ERR_ALIAS
    # filter writing into its own input
    assert lib.arbor_filterLighting(A, A + 4 * MB, A + 8 * MB, A, A + 12 * MB, 64, 64, None) == ab.ERR_ALIAS


def test_read_only_aliasing_allowed_until_launch(lib):
    """Two read-only bindings may share a buffer (runtime.js:325 rejects only
    writable aliasing): with width 0 the call validates and returns without a
    launch."""
    assert lib.arbor_tracePixels(A, A, A + 8 * MB, A + 9 * MB, A + 16 * MB, 0, 64, None) == ab.OK


def test_scalar_ranges(lib):
    assert lib.arbor_sortPass(A, A + MB, 32768, 2, None) == ab.ERR_VALUE
    assert lib.arbor_sortPass(A, A + MB, -1, 2, None) == ab.ERR_VALUE
    assert lib.arbor_reduceBounds(A, 16385, None) == ab.ERR_VALUE
    assert lib.arbor_reduceBounds(A, -1, None) == ab.ERR_VALUE
    assert lib.arbor_reduceBounds(A, 0, None) == ab.OK  # nothing to reduce: no launch
    assert lib.arbor_updateCamera(A, A + MB, A + 2 * MB, float("nan"), 64, 64, None) == ab.ERR_VALUE
    assert lib.arbor_updateCamera(A, A + MB, A + 2 * MB, float("inf"), 64, 64, None) == ab.ERR_VALUE
    # C[9] is a float: sample indices beyond 2^24 are not representable
    assert lib.arbor_setSample(A, -1, 0, None) == ab.ERR_VALUE
    assert lib.arbor_setSample(A, (1 << 24) + 1, 0, None) == ab.ERR_VALUE
    assert lib.arbor_setSample(None, 0, 1, None) == ab.ERR_NULL


def test_image_sizes(lib):
    args = (A, A + 4 * MB, A + 8 * MB, A + 9 * MB, A + 16 * MB)
    assert lib.arbor_tracePixels(*args, -1, 64, None) == ab.ERR_VALUE
    assert lib.arbor_tracePixels(*args, 64, 0, None) == ab.OK  # zero workgroups: no-op
    assert lib.arbor_tracePixels(*args, 65536 * 8 + 1, 8, None) == ab.ERR_LIMIT  # > 65535 workgroups
    assert lib.arbor_resolvePixels(A, A + 4 * MB, A + 8 * MB, A + 9 * MB, 30000, 30000, None) == ab.ERR_LIMIT


def test_engine_rejections_without_device(lib):
    h = ctypes.c_void_p()
    st = lib.arbor_engine_create(ctypes.byref(h), 640, 360, 1, 0, None)
    if lib.arbor_device_ready():
        pytest.skip("a device is present; covered by the GPU engine tests")
    assert st == ab.ERR_NO_DEVICE and not h.value
    assert lib.arbor_engine_create(None, 640, 360, 1, 0, None) == ab.ERR_NULL
    assert lib.arbor_engine_frame(None, 0.016) == ab.ERR_NULL
    assert lib.arbor_engine_destroy(None) == ab.OK


def test_denoiser_rejections_without_device(lib):
    """Null handles are rejected by every denoiser entry that takes one,
    before any device work; the loss kinds are ARBOR_LOSS_L1 and L2."""
    assert lib.arbor_denoiser_set_loss(None, ab.LOSS_L1) == ab.ERR_NULL
    assert "NULL" in ab.last_error()
    assert lib.arbor_denoiser_set_backend(None, 1) == ab.ERR_NULL
    header = open(HEADER).read()
    assert re.search(r"#define ARBOR_LOSS_L1 0\b", header) and re.search(r"#define ARBOR_LOSS_L2 1\b", header)
    assert (ab.LOSS_L1, ab.LOSS_L2) == (0, 1)


def test_launch_counter_starts_without_launches(lib):
    assert lib.arbor_launch_count() >= 0


def test_batch_rejections_without_device(lib):
    """Batch arguments are checked before any device work."""
    import ctypes

    import workloads

    h = ctypes.c_void_p()
    views = (ab.BatchView * 2)()
    for v in views:
        v.scene, v.width, v.height = 0, 64, 32
        v.C[:] = [float(x) for x in workloads.view_pose_state(7, 64, 32, 0.0, 0.0, 0.0, 0.0)]
    seeds = (ctypes.c_int * 2)(7, 1788)
    assert lib.arbor_batch_create(None, seeds, 2, views, 2, None) == ab.ERR_NULL
    assert lib.arbor_batch_create(ctypes.byref(h), seeds, 2, views, 0, None) == ab.ERR_VALUE
    assert lib.arbor_batch_create(ctypes.byref(h), seeds, 0, views, 2, None) == ab.ERR_VALUE
    bad_seeds = (ctypes.c_int * 2)(7, 1000001)
    assert lib.arbor_batch_create(ctypes.byref(h), bad_seeds, 2, views, 2, None) == ab.ERR_VALUE
    views[1].scene = 2
    assert lib.arbor_batch_create(ctypes.byref(h), seeds, 2, views, 2, None) == ab.ERR_VALUE
    assert b"scene 2" in lib.arbor_last_error()
    views[1].scene, views[1].width = 1, 0
    assert lib.arbor_batch_create(ctypes.byref(h), seeds, 2, views, 2, None) == ab.ERR_VALUE
    views[1].width = 64
    views[1].C[5] = float("nan")
    assert lib.arbor_batch_create(ctypes.byref(h), seeds, 2, views, 2, None) == ab.ERR_VALUE
    views[1].C[5] = 0.0
    views[1].width = 65536 * 8 + 1
    assert lib.arbor_batch_create(ctypes.byref(h), seeds, 2, views, 2, None) == ab.ERR_LIMIT
    views[1].width = 64
    assert lib.arbor_batch_create(ctypes.byref(h), seeds, 2, views, 2, None) == ab.ERR_NO_DEVICE
    assert lib.arbor_batch_render(None) == ab.ERR_NULL
    assert lib.arbor_batch_destroy(None) == ab.OK


def test_image_files(lib, tmp_path):
    """PPM bytes equal the reference harness's own writer (Renderer::save,
    tests/native_harness.cpp:53) when its build is present; PFM layout."""
    import ctypes

    import numpy as np

    w, h = 7, 3
    px = (np.arange(w * h, dtype=np.uint32) * 2654435761).astype(np.uint32) | np.uint32(0xFF000000)
    ppm = tmp_path / "a.ppm"
    assert lib.arbor_write_ppm(str(ppm).encode(), px.ctypes.data, w, h) == ab.OK
    data = ppm.read_bytes()
    rgb = np.stack([px & 255, (px >> 8) & 255, (px >> 16) & 255], 1).astype(np.uint8).tobytes()
    assert data == f"P6\n{w} {h}\n255\n".encode() + rgb
    ref_so = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libarbor_ref.so")
    if os.path.exists(ref_so):
        ref = ctypes.CDLL(ref_so)
        if hasattr(ref, "oracle_harnessSave"):
            ref.oracle_harnessSave.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
            out = tmp_path / "ref.ppm"
            ref.oracle_harnessSave(px.ctypes.data, w, h, str(out).encode())
            assert out.read_bytes() == data
    img = np.random.default_rng(0).random(w * h * 4).astype(np.float32)
    pfm = tmp_path / "a.pfm"
    assert lib.arbor_write_pfm(str(pfm).encode(), img.ctypes.data, w, h) == ab.OK
    raw = pfm.read_bytes()
    head = f"PF\n{w} {h}\n-1.0\n".encode()
    assert raw.startswith(head)
    body = np.frombuffer(raw[len(head):], "<f4").reshape(h, w, 3)
    assert np.array_equal(body[::-1], img.reshape(h, w, 4)[..., :3])
    assert lib.arbor_write_ppm(None, px.ctypes.data, w, h) == ab.ERR_NULL
    assert lib.arbor_write_ppm(str(ppm).encode(), px.ctypes.data, 0, h) == ab.ERR_VALUE


def test_in_order_entries_validate_like_the_batched_ones(lib):
    """The in-order trace/shade take tracePixels'/shadePixels' buffers and
    reject the same bad bindings before any launch."""
    args = (A, A + 4 * MB, A + 8 * MB, A + 9 * MB, A + 16 * MB)
    assert lib.arbor_tracePixelsInOrder(None, *args[1:], 64, 64, 0, None) == ab.ERR_NULL
    assert lib.arbor_tracePixelsInOrder(A + 4, *args[1:], 64, 64, 0, None) == ab.ERR_ALIGN
    assert lib.arbor_tracePixelsInOrder(A, A + 4 * MB, A + 8 * MB, A + 9 * MB, A + 64, 64, 64, 0, None) == ab.ERR_ALIAS
    assert lib.arbor_tracePixelsInOrder(*args, -1, 64, 0, None) == ab.ERR_VALUE
    assert lib.arbor_tracePixelsInOrder(*args, 64, 0, 1, None) == ab.OK  # zero workgroups: no-op
    shade = (A, A + 4 * MB, A + 8 * MB, A + 9 * MB, A + 16 * MB, A + 32 * MB, A + 48 * MB)
    assert lib.arbor_shadePixelsInOrder(*shade[:6], None, 64, 64, 0, None) == ab.ERR_NULL
    assert lib.arbor_shadePixelsInOrder(*shade[:5], A + 32 * MB, A + 32 * MB, 64, 64, 0, None) == ab.ERR_ALIAS
    assert lib.arbor_shadePixelsInOrder(*shade, 64, 0, 0, None) == ab.OK
