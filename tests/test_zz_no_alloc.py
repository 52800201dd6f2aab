"""arbor_sortKeysNoAlloc: the sort for callers that cannot allocate device
memory (a host that owns every buffer and binds only the ABI records, or a
frame loop under a fixed memory budget).  It must give exactly what
arbor_sortKeys gives, call after call, although every call reuses the same
library-owned scratch array and that array still holds the previous call's
data.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gu():
    import gpu_util

    return gpu_util


def sort_with_scratch(cuda, gu, raw):
    keys, order = gu.dev(raw), gu.dev(np.arange(len(raw), dtype=np.uint32))
    gu.ok(cuda.call("arbor_sortKeys", keys, order, gu.zeros_u(2 * 32768)))
    return gu.host(keys, np.uint32), gu.host(order, np.uint32)


def sort_no_alloc(cuda, gu, raw, count=None):
    keys, order = gu.dev(raw), gu.dev(np.arange(len(raw), dtype=np.uint32))
    gu.ok(cuda.call("arbor_sortKeysNoAlloc", keys, order, len(raw) if count is None else count))
    return gu.host(keys, np.uint32), gu.host(order, np.uint32)


def test_matches_sort_with_scratch_two_calls_in_a_row(cuda, oracle, gu):
    scene = oracle.build_scene(1788)
    rng = np.random.default_rng(11)
    first = scene["RawKeys"].copy()
    second = rng.integers(0, 2**32, 32768, dtype=np.uint64).astype(np.uint32)
    for raw in (first, second):  # the second call finds the first call's data in the array
        k_ref, o_ref = sort_with_scratch(cuda, gu, raw)
        k, o = sort_no_alloc(cuda, gu, raw)
        assert np.array_equal(k, k_ref)
        assert np.array_equal(o, o_ref)
    assert np.array_equal(sort_no_alloc(cuda, gu, first)[1], scene["Order"])


def test_partial_count_and_limits(cuda, gu):
    rng = np.random.default_rng(12)
    raw = rng.integers(0, 1 << 30, 5000, dtype=np.uint64).astype(np.uint32)
    k, o = sort_no_alloc(cuda, gu, raw)
    want = np.lexsort((np.arange(5000), raw))
    assert np.array_equal(o, want.astype(np.uint32)) and np.array_equal(k, raw[want])
    import arbor_b200 as ab

    big = gu.zeros_u(32769)
    assert ab.call("arbor_sortKeysNoAlloc", big, gu.zeros_u(32769), 32769) == ab.ERR_LIMIT
    assert "32768" in ab.last_error()
    assert ab.call("arbor_sortKeysNoAlloc", big, gu.zeros_u(32769), -1) == ab.ERR_VALUE
    assert ab.call("arbor_sortKeysNoAlloc", big, big, 0) == ab.OK
