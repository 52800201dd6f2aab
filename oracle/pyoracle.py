"""TEST INFRASTRUCTURE ONLY - ctypes driver for the CPU oracle libraries.

Loads either oracle/liboracle.so (the plain-C restatement, float),
oracle/liboracle64.so (the same restatement in double: the FP64 rerun) or
oracle/_ref/libarbor_ref.so (the reference's own harness code built from its
sources).  All three export the same ``oracle_*`` symbols.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: $ARBOR_REFERENCE_DIR, else a directory named
# "reference" beside this repository's root.
REFERENCE_DIR = os.environ.get("ARBOR_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")

CAPACITY = 32768
NODE_COUNT = 65536
PS = 24
CS = 20
CURVES = 2109
WOOD_COUNT = 5124
LEAF_COUNT = 24192
ROCK_COUNT = 96
OBJECT_COUNT = 29412
GROW_COUNTS = (9, 12, 72, 288, 1728)

_f = ctypes.POINTER(ctypes.c_float)
_u = ctypes.POINTER(ctypes.c_uint32)
_i = ctypes.POINTER(ctypes.c_int)
_c_int = ctypes.c_int
_c_float = ctypes.c_float

_SIGNATURES = {
    "oracle_is_f64": (_c_int, []),
    "oracle_set_threads": (None, [_c_int]),
    "oracle_max_threads": (_c_int, []),
    "oracle_growTree": (None, [_f, _c_int, _c_int]),
    "oracle_makePrimitives": (None, [_f, _f, _c_int]),
    "oracle_makeKeys": (None, [_f, _u, _u]),
    "oracle_sortPass": (None, [_u, _u, _c_int, _c_int]),
    "oracle_sortPairs": (None, [_u, _u, _c_int]),
    "oracle_makeBounds": (None, [_f, _u, _f]),
    "oracle_reduceBounds": (None, [_f, _c_int]),
    "oracle_initCamera": (None, [_f, _f, _c_int]),
    "oracle_updateCamera": (None, [_f, _f, _f, _c_float, _c_int, _c_int]),
    "oracle_tracePixels": (None, [_f, _f, _u, _f, _f, _c_int, _c_int, _c_int, _c_int, _c_int]),
    "oracle_shadePixels": (None, [_f, _f, _u, _f, _f, _f, _f, _c_int, _c_int, _c_int, _c_int, _c_int]),
    "oracle_filterLighting": (None, [_f, _f, _f, _f, _f, _c_int, _c_int, _c_int, _c_int]),
    "oracle_resolvePixels": (None, [_f, _f, _u, _f, _c_int, _c_int, _c_int, _c_int]),
    "oracle_tracePixelList": (None, [_f, _f, _u, _f, _f, _c_int, _c_int, _i, _c_int, _c_int]),
    "oracle_traceTreeRay": (None, [_f, _f, _u, _f, _f, _c_float, _c_float, _c_float, _c_float, _c_int, _c_int, _f]),
    "oracle_objectT": (_c_float, [_f, _c_int, _f, _f, _c_float, _c_float, _c_float, _c_int]),
    "oracle_leafT": (_c_float, [_f, _c_int, _f, _f, _c_float, _c_float, _c_float]),
    "oracle_boxSpan": (None, [_f, _f, _f, _f, _f]),
    "oracle_bounds": (None, [_f, _c_int, _f, _f]),
    "oracle_barkCut": (_c_float, [_f, _c_int, _f, _c_float]),
    "oracle_bandWeight": (_c_float, [_c_float, _c_float]),
    "oracle_rnd": (_c_float, [_c_int, _c_int]),
    "oracle_forestSeed": (_c_int, [_c_int, _c_int]),
    "oracle_forestInstance": (None, [_c_int, _c_int, _f]),
    "oracle_exhaustiveRay": (None, [_f, _f, _f, _c_float, _f]),
    "oracle_harnessRay": (None, [_c_int, _f, _f]),
    "oracle_footprintSweep": (None, [_f, _c_int, _f]),
    "oracle_leafPair": (None, [_f, _c_int, _f]),
    "oracle_frameRows": (None, [_f, _f, _u, _f, _f, _f, _f, _f, _f, _u, _c_int, _c_int, _i, _c_int, _c_int]),
}
_OPTIONAL = {
    # only in the reference build: the harness's Renderer constructor
    "oracle_harnessBuild": (None, [_c_int, _f, _f, _u, _u, _f]),
    # only in the port: shadePixels' shading normal per pixel, and the forest
    # of several species (no reference counterpart)
    "oracle_shadeNormals": (None, [_f, _f, _f, _f, _c_int, _c_int, _c_int, _c_int, _c_int]),
    "oracle_tracePixelsSpecies": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i, _f, _f, _c_int, _c_int, _c_int, _c_int]),
    "oracle_shadePixelsSpecies": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i, _f, _f, _f, _f, _c_int, _c_int, _c_int,
                                         _c_int]),
}


def _p(a: np.ndarray):
    if a.dtype == np.float32:
        return a.ctypes.data_as(_f)
    if a.dtype == np.uint32:
        return a.ctypes.data_as(_u)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_i)
    raise TypeError(a.dtype)


def _v(x):
    return _p(np.ascontiguousarray(np.asarray(x, dtype=np.float32)))


def library_path(kind: str) -> str:
    return {
        "port": os.path.join(HERE, "liboracle.so"),
        "port64": os.path.join(HERE, "liboracle64.so"),
        "reference": os.path.join(HERE, "_ref", "libarbor_ref.so"),
    }[kind]


def build(kind: str = "port") -> str:
    """Compile the requested oracle library with oracle/Makefile if missing."""
    path = library_path(kind)
    if os.path.exists(path):
        return path
    target = "ref" if kind == "reference" else "all"
    if kind == "reference" and not os.path.isdir(REFERENCE_DIR):
        raise FileNotFoundError("reference sources not present; oracle/_ref cannot be built here")
    subprocess.run(["make", "-s", "-C", HERE, target, f"REF={REFERENCE_DIR}"], check=True)
    return path


def available(kind: str) -> bool:
    try:
        build(kind)
        return True
    except Exception:
        return False


class Oracle:
    """One oracle library; the methods mirror the 12 reference entry points."""

    def __init__(self, kind: str = "port"):
        self.kind = kind
        self.path = build(kind)
        self.lib = ctypes.CDLL(self.path)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(self.lib, name, None)
            if fn is None:
                raise AttributeError(f"{self.path} lacks {name}")
            fn.restype = res
            fn.argtypes = args
        self.has_harness_build = hasattr(self.lib, "oracle_harnessBuild")
        for name, (res, args) in _OPTIONAL.items():
            fn = getattr(self.lib, name, None)
            if fn is not None:
                fn.restype = res
                fn.argtypes = args
        self.is_f64 = bool(self.lib.oracle_is_f64())

    # -- threads
    def set_threads(self, n: int) -> None:
        self.lib.oracle_set_threads(int(n))

    def max_threads(self) -> int:
        return int(self.lib.oracle_max_threads())

    # -- scene build (the harness's Renderer constructor, native_harness.cpp:45-48)
    def build_scene(self, seed: int, bitonic: bool = False) -> dict:
        B = np.zeros(CURVES * CS, np.float32)
        P = np.zeros(CAPACITY * PS, np.float32)
        keys = np.zeros(CAPACITY, np.uint32)
        order = np.zeros(CAPACITY, np.uint32)
        nodes = np.zeros(NODE_COUNT * 8, np.float32)
        for level in range(5):
            self.lib.oracle_growTree(_p(B), level, seed)
        self.lib.oracle_makePrimitives(_p(B), _p(P), seed)
        self.lib.oracle_makeKeys(_p(P), _p(keys), _p(order))
        raw_keys = keys.copy()
        if bitonic:
            self.bitonic(keys, order)
        else:
            self.lib.oracle_sortPairs(_p(keys), _p(order), CAPACITY)
        self.lib.oracle_makeBounds(_p(P), _p(order), _p(nodes))
        first = CAPACITY // 2
        while first >= 1:
            self.lib.oracle_reduceBounds(_p(nodes), first)
            first //= 2
        return {"seed": seed, "B": B, "P": P, "Keys": keys, "Order": order, "Nodes": nodes, "RawKeys": raw_keys}

    def grow(self, B, level, seed):
        self.lib.oracle_growTree(_p(B), level, seed)

    def make_primitives(self, B, P, seed):
        self.lib.oracle_makePrimitives(_p(B), _p(P), seed)

    def make_keys(self, P, keys, order):
        self.lib.oracle_makeKeys(_p(P), _p(keys), _p(order))

    def sort_pass(self, keys, order, distance, span):
        self.lib.oracle_sortPass(_p(keys), _p(order), distance, span)

    def bitonic(self, keys, order):
        span = 2
        while span <= CAPACITY:
            d = span // 2
            while d > 0:
                self.lib.oracle_sortPass(_p(keys), _p(order), d, span)
                d //= 2
            span *= 2

    def sort_pairs(self, keys, order):
        self.lib.oracle_sortPairs(_p(keys), _p(order), len(keys))

    def make_bounds(self, P, order, nodes):
        self.lib.oracle_makeBounds(_p(P), _p(order), _p(nodes))

    def reduce_bounds(self, nodes, first):
        self.lib.oracle_reduceBounds(_p(nodes), first)

    # -- camera
    def init_camera(self, P, seed) -> np.ndarray:
        C = np.zeros(64, np.float32)
        self.lib.oracle_initCamera(_p(C), _p(P), seed)
        return C

    def update_camera(self, C, I, P, delta, w, h):
        self.lib.oracle_updateCamera(_p(C), _p(I), _p(P), float(delta), w, h)

    # -- image passes
    def trace(self, scene, C, w, h, y0=0, y1=None, single=False, Hit=None):
        y1 = h if y1 is None else y1
        Hit = np.zeros(w * h * 4, np.float32) if Hit is None else Hit
        self.lib.oracle_tracePixels(_p(scene["P"]), _p(scene["Nodes"]), _p(scene["Order"]), _p(C), _p(Hit), w, h, y0, y1, int(single))
        return Hit

    def shade(self, scene, C, Hit, w, h, y0=0, y1=None, single=False, Linear=None, Guide=None):
        y1 = h if y1 is None else y1
        Linear = np.zeros(w * h * 4, np.float32) if Linear is None else Linear
        Guide = np.zeros(w * h * 4, np.float32) if Guide is None else Guide
        self.lib.oracle_shadePixels(_p(scene["P"]), _p(scene["Nodes"]), _p(scene["Order"]), _p(C), _p(Hit), _p(Linear), _p(Guide), w, h, y0, y1, int(single))
        return Linear, Guide

    def shade_normals(self, scene, C, Hit, w, h, y0=0, y1=None, single=False, Normal=None):
        """shadePixels' shading normal per pixel (world space, facing the camera; zero for sky)."""
        y1 = h if y1 is None else y1
        Normal = np.zeros(w * h * 4, np.float32) if Normal is None else Normal
        self.lib.oracle_shadeNormals(_p(scene["P"]), _p(C), _p(Hit), _p(Normal), w, h, y0, y1, int(single))
        return Normal

    @staticmethod
    def _species_tables(scenes: list, of):
        keep = [np.ascontiguousarray(s[k]) for s in scenes for k in ("P", "Nodes", "Order")]
        ptr = lambda key: (ctypes.c_void_p * len(scenes))(*[s[key].ctypes.data for s in scenes])  # noqa: E731
        of = np.ascontiguousarray(of, dtype=np.int32)
        assert of.shape == (324,) and of.min() >= 0 and of.max() < len(scenes)
        return ptr("P"), ptr("Nodes"), ptr("Order"), of, keep

    def trace_species(self, scenes: list, of, C, w, h, y0=0, y1=None, Hit=None):
        """tracePixels over a forest whose instance t uses scenes[of[t]]."""
        y1 = h if y1 is None else y1
        Hit = np.zeros(w * h * 4, np.float32) if Hit is None else Hit
        P, N, O, of, _keep = self._species_tables(scenes, of)
        self.lib.oracle_tracePixelsSpecies(P, N, O, _p(of), _p(C), _p(Hit), w, h, y0, y1)
        return Hit

    def shade_species(self, scenes: list, of, C, Hit, w, h, y0=0, y1=None, Linear=None, Guide=None):
        """shadePixels over a forest whose instance t uses scenes[of[t]]."""
        y1 = h if y1 is None else y1
        Linear = np.zeros(w * h * 4, np.float32) if Linear is None else Linear
        Guide = np.zeros(w * h * 4, np.float32) if Guide is None else Guide
        P, N, O, of, _keep = self._species_tables(scenes, of)
        self.lib.oracle_shadePixelsSpecies(P, N, O, _p(of), _p(C), _p(Hit), _p(Linear), _p(Guide), w, h, y0, y1)
        return Linear, Guide

    def filter(self, Linear, Guide, Hit, C, w, h, y0=0, y1=None, Filtered=None):
        y1 = h if y1 is None else y1
        Filtered = np.zeros(w * h * 4, np.float32) if Filtered is None else Filtered
        self.lib.oracle_filterLighting(_p(Linear), _p(Guide), _p(Hit), _p(Filtered), _p(C), w, h, y0, y1)
        return Filtered

    def resolve(self, Filtered, History, C, w, h, y0=0, y1=None, Pixels=None):
        y1 = h if y1 is None else y1
        Pixels = np.zeros(w * h, np.uint32) if Pixels is None else Pixels
        self.lib.oracle_resolvePixels(_p(Filtered), _p(History), _p(Pixels), _p(C), w, h, y0, y1)
        return Pixels

    def frame(self, scene, C, w, h, History=None, single=False) -> dict:
        """trace -> shade -> filter -> resolve (native_harness.cpp:52)."""
        History = np.zeros(w * h * 4, np.float32) if History is None else History
        Hit = self.trace(scene, C, w, h, single=single)
        Linear, Guide = self.shade(scene, C, Hit, w, h, single=single)
        Filtered = self.filter(Linear, Guide, Hit, C, w, h)
        Pixels = self.resolve(Filtered, History, C, w, h)
        return {"Hit": Hit, "Linear": Linear, "Guide": Guide, "Filtered": Filtered, "History": History, "Pixels": Pixels}

    def frame_rows(self, scene, C, w, h, rows, bufs: dict, single=False) -> None:
        """trace, shade, filter, resolve over the listed rows only (into bufs)."""
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        self.lib.oracle_frameRows(_p(scene["P"]), _p(scene["Nodes"]), _p(scene["Order"]), _p(C), _p(bufs["Hit"]), _p(bufs["Linear"]),
                                  _p(bufs["Guide"]), _p(bufs["Filtered"]), _p(bufs["History"]), _p(bufs["Pixels"]), w, h, _p(rows),
                                  len(rows), int(single))

    def trace_pixel_list(self, scene, C, w, h, xy: np.ndarray, single=False) -> np.ndarray:
        """Trace only the listed (x, y) pixels; returns a full-size Hit with the rest zero."""
        xy = np.ascontiguousarray(xy, dtype=np.int32).reshape(-1)
        Hit = np.zeros(w * h * 4, np.float32)
        self.lib.oracle_tracePixelList(_p(scene["P"]), _p(scene["Nodes"]), _p(scene["Order"]), _p(C), _p(Hit), w, h, _p(xy), len(xy) // 2, int(single))
        return Hit

    # -- function-level probes
    def trace_tree_ray(self, scene, ro, rd, cone, time=0.0, wind=0.0, best=1e5, ignore=-1, shadows=False):
        out = np.zeros(2, np.float32)
        self.lib.oracle_traceTreeRay(_p(scene["P"]), _p(scene["Nodes"]), _p(scene["Order"]), _v(ro), _v(rd), cone, time, wind, best, ignore, int(shadows), _p(out))
        return float(out[0]), int(out[1])

    def object_t(self, P, oid, ro, rd, fp, time=0.0, wind=0.0, refine=True):
        return float(self.lib.oracle_objectT(_p(P), oid, _v(ro), _v(rd), fp, time, wind, int(refine)))

    def leaf_t(self, P, oid, ro, rd, fp, time=0.0, wind=0.0):
        return float(self.lib.oracle_leafT(_p(P), oid, _v(ro), _v(rd), fp, time, wind))

    def box_span(self, ro, rd, lo, hi):
        out = np.zeros(2, np.float32)
        self.lib.oracle_boxSpan(_v(ro), _v(rd), _v(lo), _v(hi), _p(out))
        return float(out[0]), float(out[1])

    def bounds(self, P, oid):
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        self.lib.oracle_bounds(_p(P), oid, _p(lo), _p(hi))
        return lo, hi

    def bark_cut(self, P, oid, p, fp):
        return float(self.lib.oracle_barkCut(_p(P), oid, _v(p), fp))

    def band_weight(self, period, fp):
        return float(self.lib.oracle_bandWeight(period, fp))

    def rnd(self, n, seed):
        return float(self.lib.oracle_rnd(n, seed))

    def forest_seed(self, tree, ws):
        return int(self.lib.oracle_forestSeed(tree, ws))

    def exhaustive_ray(self, P, ro, rd, cone):
        out = np.zeros(2, np.float32)
        self.lib.oracle_exhaustiveRay(_p(P), _v(ro), _v(rd), cone, _p(out))
        return float(out[0]), int(out[1])

    def harness_ray(self, ray: int):
        ro = np.zeros(3, np.float32)
        rd = np.zeros(3, np.float32)
        self.lib.oracle_harnessRay(ray, _p(ro), _p(rd))
        return ro, rd

    def footprint_sweep(self, P, oid: int = 4):
        out = np.zeros(3, np.float32)
        self.lib.oracle_footprintSweep(_p(P), oid, _p(out))
        return float(out[0]), bool(out[1]), bool(out[2])

    def leaf_pair(self, P, k: int):
        out = np.zeros(2, np.float32)
        self.lib.oracle_leafPair(_p(P), k, _p(out))
        return float(out[0]), float(out[1])

    def harness_build(self, seed: int) -> dict:
        """The reference harness's own Renderer(seed) buffers (reference build only)."""
        B = np.zeros(CURVES * CS, np.float32)
        P = np.zeros(CAPACITY * PS, np.float32)
        keys = np.zeros(CAPACITY, np.uint32)
        order = np.zeros(CAPACITY, np.uint32)
        nodes = np.zeros(NODE_COUNT * 8, np.float32)
        self.lib.oracle_harnessBuild(seed, _p(B), _p(P), _p(keys), _p(order), _p(nodes))
        return {"seed": seed, "B": B, "P": P, "Keys": keys, "Order": order, "Nodes": nodes}

    def forest_instance(self, tree, ws):
        out = np.zeros(6, np.float32)
        self.lib.oracle_forestInstance(tree, ws, _p(out))
        return out
