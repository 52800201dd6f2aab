"""A forest of several species on the GPU against the oracle.

arbor_traceSpeciesPixels / arbor_shadeSpeciesPixels trace and shade the
reference's 324-instance forest with per-instance geometry: instance t takes
its records and BVH from scene species_of[t] of a set of scenes held back to
back (the reference keeps one resident tree for every instance, README.md:8).
The oracle composes the reference's traceTree per instance the same way
(oracle_tracePixelsSpecies / oracle_shadePixelsSpecies).

Bars: with one species the entries equal arbor_tracePixels /
arbor_shadePixels bit for bit; with several, the comparison contract of the
single-scene forest (IDs on >= 99.9 % of pixels, t within 2e-3 m + 1e-4 t on
>= 99.95 % of agreeing hits, Linear within 2e-3 on >= 99.9 % of pixels shaded
from the same Hit).
"""
import ctypes

import numpy as np
import pytest

from conftest import u32

pytestmark = pytest.mark.gpu
WS = 7
SEEDS = (7, 1, 42)


@pytest.fixture(scope="module")
def gu():
    import gpu_util

    return gpu_util


def species_of(n: int) -> np.ndarray:
    import workloads

    return workloads.species_of(n, WS)


def preset_camera(oracle, scene, view, w, h, shadows):
    C = oracle.init_camera(scene["P"], WS)
    I = np.zeros(32, np.float32)
    I[5] = view
    oracle.update_camera(C, I, scene["P"], 1.0 / 60, w, h)
    C[22] = 1.0 if shadows else 0.0
    return C


def arena(gu, scenes):
    """The scenes' P, Nodes and Order back to back on the device."""
    return {k: gu.dev(np.concatenate([s[k] for s in scenes])) for k in ("P", "Nodes", "Order")}


def call_species(cuda, a, n, of, entry, *rest):
    of = np.ascontiguousarray(of, np.int32)
    return cuda.call(entry, a["P"], a["Nodes"], a["Order"], n, of.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), *rest)


def test_one_species_equals_the_forest(cuda, gu, scenes, oracle):
    w, h = 320, 192
    s = scenes(7)
    a = arena(gu, [s])
    one = gu.DevScene(s)
    for view, shadows in ((1, True), (2, False), (4, True)):
        C = gu.dev(preset_camera(oracle, s, view, w, h, shadows))
        hit, hit_ref = gu.zeros_f(w * h * 4), gu.zeros_f(w * h * 4)
        gu.ok(call_species(cuda, a, 1, np.zeros(324), "arbor_traceSpeciesPixels", C, hit, w, h))
        gu.ok(cuda.call("arbor_tracePixels", one.P, one.Nodes, one.Order, C, hit_ref, w, h))
        assert np.array_equal(u32(gu.host(hit)), u32(gu.host(hit_ref)))
        lin, gui, lin_ref, gui_ref = (gu.zeros_f(w * h * 4) for _ in range(4))
        gu.ok(call_species(cuda, a, 1, np.zeros(324), "arbor_shadeSpeciesPixels", C, hit, lin, gui, w, h))
        gu.ok(cuda.call("arbor_shadePixels", one.P, one.Nodes, one.Order, C, hit, lin_ref, gui_ref, w, h))
        assert np.array_equal(u32(gu.host(lin)), u32(gu.host(lin_ref)))
        assert np.array_equal(u32(gu.host(gui)), u32(gu.host(gui_ref)))


@pytest.mark.parametrize("view,shadows", [(1, False), (2, True), (3, True), (5, False)])
def test_three_species_against_oracle(cuda, gu, scenes, oracle, view, shadows):
    w, h = 240, 160
    sc = [scenes(seed) for seed in SEEDS]
    of = species_of(len(sc))
    a = arena(gu, sc)
    C = preset_camera(oracle, sc[0], view, w, h, shadows)
    dC = gu.dev(C)
    hit = gu.zeros_f(w * h * 4)
    gu.ok(call_species(cuda, a, len(sc), of, "arbor_traceSpeciesPixels", dC, hit, w, h))
    got = gu.host(hit).reshape(-1, 4)
    want = oracle.trace_species(sc, of, C, w, h).reshape(-1, 4)
    same = (got[:, 1] == want[:, 1]) & (got[:, 2] == want[:, 2])
    both = same & (want[:, 0] < 1e5)
    t_ok = np.abs(got[both, 0] - want[both, 0]) <= 2e-3 + 1e-4 * want[both, 0]
    trees = np.unique(want[want[:, 1] >= 0, 2]).astype(int)
    print(f"[species view {view}] id agreement {same.mean():.5f}; t within tolerance {t_ok.mean():.5f}; "
          f"{len(trees)} trees hit, species {sorted(set(of[trees].tolist()))}")
    assert same.mean() >= 0.999
    assert t_ok.mean() >= 0.9995
    assert len(set(of[trees].tolist())) >= 2, "the view should see more than one species"
    # shading on the oracle's Hit
    lin_ref, gui_ref = oracle.shade_species(sc, of, C, want.reshape(-1), w, h)
    lin, gui = gu.zeros_f(w * h * 4), gu.zeros_f(w * h * 4)
    gu.ok(call_species(cuda, a, len(sc), of, "arbor_shadeSpeciesPixels", dC, gu.dev(want.reshape(-1)), lin, gui, w, h))
    L, G = gu.host(lin).reshape(-1, 4), gu.host(gui).reshape(-1, 4)
    Lr, Gr = lin_ref.reshape(-1, 4), gui_ref.reshape(-1, 4)
    errL = np.max(np.abs(L[:, :3] - Lr[:, :3]) / np.maximum(1.0, np.abs(Lr[:, :3])), 1)
    errG = np.max(np.abs(G[:, :3] - Gr[:, :3]), 1)
    print(f"[species view {view} shadows {shadows}] Linear within 2e-3 on {np.mean(errL <= 2e-3):.5f}")
    assert np.mean(errL <= 2e-3) >= 0.999
    assert np.mean(errG <= 2e-3) >= 0.999


def test_species_arguments_rejected(cuda, gu, scenes):
    import arbor_b200 as ab

    s = scenes(7)
    a = arena(gu, [s])
    C, hit = gu.zeros_f(64), gu.zeros_f(64 * 64 * 4)
    assert call_species(cuda, a, 0, np.zeros(324), "arbor_traceSpeciesPixels", C, hit, 64, 64) == ab.ERR_VALUE
    assert call_species(cuda, a, 257, np.zeros(324), "arbor_traceSpeciesPixels", C, hit, 64, 64) == ab.ERR_VALUE
    bad = np.zeros(324, np.int32)
    bad[17] = 1
    assert call_species(cuda, a, 1, bad, "arbor_traceSpeciesPixels", C, hit, 64, 64) == ab.ERR_VALUE
    assert "species_of[17]" in ab.last_error()
