"""ctypes binding of libarbor_b200.so (include/arbor.h) for tests and the benchmark.

The library is the product; this module only loads it and passes device
pointers (torch tensors are used for device memory and streams).  There is
no fallback: if the shared object is missing, importing fails loudly.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libarbor_b200.so")
HEADER = os.path.join(HERE, "..", "include", "arbor.h")

CAPACITY = 32768
NODE_COUNT = 65536
PS = 24
CS = 20
CURVES = 2109
OBJECT_COUNT = 29412
SORT_SCRATCH_WORDS = 2 * CAPACITY

STATUS = {
    0: "ARBOR_OK", 1: "ARBOR_ERR_NULL", 2: "ARBOR_ERR_VALUE", 3: "ARBOR_ERR_ALIGN", 4: "ARBOR_ERR_ALIAS",
    5: "ARBOR_ERR_LIMIT", 6: "ARBOR_ERR_CUDA", 7: "ARBOR_ERR_TIMEOUT", 8: "ARBOR_ERR_STATE", 9: "ARBOR_ERR_NO_DEVICE",
}
OK, ERR_NULL, ERR_VALUE, ERR_ALIGN, ERR_ALIAS, ERR_LIMIT, ERR_CUDA, ERR_TIMEOUT, ERR_STATE, ERR_NO_DEVICE = range(10)
LOSS_L1, LOSS_L2 = 0, 1  # arbor_denoiser_set_loss kinds

_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float


class EngineBuffers(ctypes.Structure):
    _fields_ = [(n, _vp) for n in ("B", "P", "Keys", "Order", "Nodes", "C", "I", "Hit", "Linear", "Guide", "Filtered", "History", "Pixels")]


class EngineInfo(ctypes.Structure):
    _fields_ = [
        ("width", _i), ("height", _i), ("seed", _i), ("single_tree", _i),
        ("frames", ctypes.c_uint64), ("allocated_bytes", ctypes.c_uint64), ("scene_bytes", ctypes.c_uint64),
        ("launches_per_frame", ctypes.c_uint32), ("camera", _f * 64),
        ("ms_build", _f), ("ms_visibility", _f), ("ms_lighting", _f), ("ms_resolve", _f),
    ]


class BatchView(ctypes.Structure):
    _fields_ = [("scene", _i), ("width", _i), ("height", _i), ("reserved", _i), ("C", _f * 64)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("tile_width", _i), ("ctas_per_sm", _i), ("order", _i), ("queue", _i)]

    def as_dict(self) -> dict:
        return {"tile_width": self.tile_width, "ctas_per_sm": self.ctas_per_sm, "order": self.order, "queue": self.queue}


class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("n_scenes", _i), ("n_views", _i), ("total_pixels", ctypes.c_uint64), ("allocated_bytes", ctypes.c_uint64),
        ("trace_tiles", _i), ("filter_tiles", _i), ("renders", ctypes.c_uint64), ("launches_per_render", ctypes.c_uint32),
        ("config", BatchConfig),
    ]


SIGNATURES = {
    "arbor_last_error": (ctypes.c_char_p, []),
    "arbor_status_name": (ctypes.c_char_p, [_i]),
    "arbor_device_ready": (_i, []),
    "arbor_launch_count": (ctypes.c_uint64, []),
    "arbor_growTree": (_i, [_vp, _i, _i, _vp]),
    "arbor_makePrimitives": (_i, [_vp, _vp, _i, _vp]),
    "arbor_makeKeys": (_i, [_vp, _vp, _vp, _vp]),
    "arbor_sortPass": (_i, [_vp, _vp, _i, _i, _vp]),
    "arbor_makeBounds": (_i, [_vp, _vp, _vp, _vp]),
    "arbor_reduceBounds": (_i, [_vp, _i, _vp]),
    "arbor_initCamera": (_i, [_vp, _vp, _i, _vp]),
    "arbor_updateCamera": (_i, [_vp, _vp, _vp, _f, _i, _i, _vp]),
    "arbor_setSample": (_i, [_vp, _i, _i, _vp]),
    "arbor_tracePixels": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_shadePixels": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_filterLighting": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_resolvePixels": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_sort_scratch_bytes": (ctypes.c_size_t, []),
    "arbor_sortKeys": (_i, [_vp, _vp, _vp, _vp]),
    "arbor_buildBounds": (_i, [_vp, _vp, _vp, _vp]),
    "arbor_sortKeysNoAlloc": (_i, [_vp, _vp, _i, _vp]),
    "arbor_buildScene": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "arbor_traceTreePixels": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_shadeTreePixels": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_shadeGBuffer": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_filterResolve": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_trace_work_slots": (ctypes.c_size_t, [_i, _i]),
    "arbor_forestInstances": (_i, [_i, _vp, _vp]),
    "arbor_traceSpeciesPixels": (_i, [_vp, _vp, _vp, _i, ctypes.POINTER(_i), _vp, _vp, _i, _i, _vp]),
    "arbor_shadeSpeciesPixels": (_i, [_vp, _vp, _vp, _i, ctypes.POINTER(_i), _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "arbor_tracePixelsInOrder": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp]),
    "arbor_shadePixelsInOrder": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp]),
    "arbor_traceWork": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp]),
    "arbor_shadeWork": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp]),
    "arbor_engine_create": (_i, [ctypes.POINTER(_vp), _i, _i, _i, _i, _vp]),
    "arbor_engine_generate": (_i, [_vp, _i]),
    "arbor_engine_resize": (_i, [_vp, _i, _i]),
    "arbor_engine_set_input": (_i, [_vp, ctypes.POINTER(_f)]),
    "arbor_engine_set_state": (_i, [_vp, ctypes.POINTER(_f)]),
    "arbor_engine_frame": (_i, [_vp, _f]),
    "arbor_engine_set_timing": (_i, [_vp, _i]),
    "arbor_engine_inspect": (_i, [_vp, ctypes.POINTER(EngineInfo)]),
    "arbor_engine_buffers_get": (_i, [_vp, ctypes.POINTER(EngineBuffers)]),
    "arbor_engine_read_pixels": (_i, [_vp, _vp, ctypes.c_size_t]),
    "arbor_engine_dispose": (_i, [_vp]),
    "arbor_engine_destroy": (_i, [_vp]),
    "arbor_engine_save_ppm": (_i, [_vp, ctypes.c_char_p]),
    "arbor_write_ppm": (_i, [ctypes.c_char_p, _vp, _i, _i]),
    "arbor_write_pfm": (_i, [ctypes.c_char_p, _vp, _i, _i]),
    "arbor_batch_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(_i), _i, ctypes.POINTER(BatchView), _i, _vp]),
    "arbor_batch_set_cameras": (_i, [_vp, ctypes.POINTER(_f), _i]),
    "arbor_batch_configure": (_i, [_vp, ctypes.POINTER(BatchConfig)]),
    "arbor_batch_get_config": (_i, [_vp, ctypes.POINTER(BatchConfig)]),
    "arbor_batch_autotune": (_i, [_vp, _i, ctypes.POINTER(BatchConfig), ctypes.POINTER(_f)]),
    "arbor_batch_render": (_i, [_vp]),
    "arbor_batch_profile": (_i, [_vp, ctypes.POINTER(_f)]),
    "arbor_batch_view_buffers": (_i, [_vp, _i, ctypes.POINTER(EngineBuffers)]),
    "arbor_batch_inspect": (_i, [_vp, ctypes.POINTER(BatchInfo)]),
    "arbor_batch_read_pixels": (_i, [_vp, _vp, ctypes.c_size_t]),
    "arbor_batch_destroy": (_i, [_vp]),
    "arbor_denoiser_create": (_i, [ctypes.POINTER(_vp), _i, _i, _i, ctypes.c_uint32, _vp]),
    "arbor_denoiser_param_count": (_i, [_vp, ctypes.POINTER(ctypes.c_size_t)]),
    "arbor_denoiser_get_params": (_i, [_vp, _vp, ctypes.c_size_t]),
    "arbor_denoiser_set_params": (_i, [_vp, _vp, ctypes.c_size_t]),
    "arbor_denoiser_features": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp]),
    "arbor_denoiser_train_step": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _f, ctypes.POINTER(_f)]),
    "arbor_denoiser_gradient": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _vp, ctypes.c_size_t, ctypes.POINTER(_f)]),
    "arbor_denoiser_infer": (_i, [_vp, _vp, _vp, _vp, _i, _i]),
    "arbor_denoiser_set_backend": (_i, [_vp, _i]),
    "arbor_denoiser_set_loss": (_i, [_vp, _i]),
    "arbor_denoiser_check": (_i, [_vp]),
    "arbor_denoiser_destroy": (_i, [_vp]),
    "arbor_accumulate": (_i, [_vp, _vp, ctypes.c_size_t, _f, _vp]),
}


class ArborError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run arbor-cuda_b200/build.py (no CPU fallback exists)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


def last_error() -> str:
    return lib().arbor_last_error().decode()


def check(status: int) -> None:
    if status != OK:
        raise ArborError(status, last_error())


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (or None / int passthrough)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def stream_handle(stream=None) -> int | None:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None


def call(name: str, *args, stream=None) -> int:
    """Call an entry point with torch tensors / ints / floats, current stream last."""
    conv = []
    for a in args:
        conv.append(ptr(a) if (a is None or hasattr(a, "data_ptr")) else a)
    return getattr(lib(), name)(*conv, stream_handle(stream))


def launches() -> int:
    return int(lib().arbor_launch_count())


class Engine:
    """Thin owner of an arbor_engine handle (include/arbor.h engine API)."""

    def __init__(self, width: int, height: int, seed: int = 1788, single_tree: bool = False, stream=None):
        self._lib = lib()
        h = _vp()
        check(self._lib.arbor_engine_create(ctypes.byref(h), width, height, seed, int(single_tree), stream_handle(stream)))
        self.handle = h

    def generate(self, seed: int) -> None:
        check(self._lib.arbor_engine_generate(self.handle, seed))

    def resize(self, w: int, h: int) -> None:
        check(self._lib.arbor_engine_resize(self.handle, w, h))

    def set_input(self, values) -> None:
        arr = (_f * 32)(*[float(v) for v in values])
        check(self._lib.arbor_engine_set_input(self.handle, arr))

    def set_state(self, values) -> None:
        arr = (_f * 64)(*[float(v) for v in values])
        check(self._lib.arbor_engine_set_state(self.handle, arr))

    def frame(self, dt: float = 1 / 60) -> None:
        check(self._lib.arbor_engine_frame(self.handle, dt))

    def set_timing(self, on: bool) -> None:
        check(self._lib.arbor_engine_set_timing(self.handle, int(on)))

    def inspect(self) -> EngineInfo:
        info = EngineInfo()
        check(self._lib.arbor_engine_inspect(self.handle, ctypes.byref(info)))
        return info

    def buffers(self) -> EngineBuffers:
        b = EngineBuffers()
        check(self._lib.arbor_engine_buffers_get(self.handle, ctypes.byref(b)))
        return b

    def read_pixels_into(self, host_ptr: int, count: int) -> None:
        check(self._lib.arbor_engine_read_pixels(self.handle, host_ptr, count))

    def dispose(self) -> None:
        check(self._lib.arbor_engine_dispose(self.handle))

    def close(self) -> None:
        if self.handle:
            self._lib.arbor_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Owner of an arbor_batch handle (include/arbor.h batched rendering).

    views: (scene index, width, height, C[64]) per view."""

    def __init__(self, seeds, views, stream=None):
        self._lib = lib()
        self.views = list(views)
        arr = (BatchView * len(self.views))()
        for i, (scene, w, h, C) in enumerate(self.views):
            arr[i].scene, arr[i].width, arr[i].height = int(scene), int(w), int(h)
            arr[i].C[:] = [float(x) for x in C]
        sd = (_i * len(seeds))(*[int(s) for s in seeds])
        h = _vp()
        check(self._lib.arbor_batch_create(ctypes.byref(h), sd, len(seeds), arr, len(self.views), stream_handle(stream)))
        self.handle = h

    def _call(self, name, *args):
        check(getattr(self._lib, name)(self.handle, *args))

    def render(self) -> None:
        self._call("arbor_batch_render")

    def profile(self) -> list[float]:
        ms = (_f * 4)()
        self._call("arbor_batch_profile", ms)
        return list(ms)

    def configure(self, tile_width: int, ctas_per_sm: int, order: int, queue: int) -> None:
        self._call("arbor_batch_configure", ctypes.byref(BatchConfig(tile_width, ctas_per_sm, order, queue)))

    def config(self) -> dict:
        c = BatchConfig()
        self._call("arbor_batch_get_config", ctypes.byref(c))
        return c.as_dict()

    def autotune(self, sample_views: int = 0) -> tuple[dict, list[float]]:
        best, ms = BatchConfig(), (_f * 16)()
        self._call("arbor_batch_autotune", sample_views, ctypes.byref(best), ms)
        return best.as_dict(), list(ms)

    def set_cameras(self, C) -> None:
        import numpy as np

        flat = np.ascontiguousarray(C, np.float32).reshape(-1)
        self._call("arbor_batch_set_cameras", flat.ctypes.data_as(ctypes.POINTER(_f)), flat.size // 64)

    def inspect(self) -> BatchInfo:
        info = BatchInfo()
        self._call("arbor_batch_inspect", ctypes.byref(info))
        return info

    def buffers(self, view: int) -> EngineBuffers:
        b = EngineBuffers()
        self._call("arbor_batch_view_buffers", view, ctypes.byref(b))
        return b

    def read_pixels_into(self, host_ptr: int, count: int) -> None:
        self._call("arbor_batch_read_pixels", host_ptr, count)

    def close(self) -> None:
        if self.handle:
            self._lib.arbor_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
