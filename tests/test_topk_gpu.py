"""Top-k by radix selection (am_top_k_ex): for every k the answer must be the first k indices of the
stable argsort with the same options (include/arrowmetal.h:1345-1350) -- value rows in key order with
ties in row order, then NaN-block and null rows in row order (or those first, nulls at the start)."""
import zlib

import numpy as np
import pyarrow as pa
import pytest

from conftest import build_array

pytestmark = pytest.mark.gpu

PLACEMENTS = ("at_end", "at_start")
ORDERS = ("ieee", "total", "nan_largest")


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def column(rng, kind, n):
    valid = rng.random(n) > 0.1
    if kind == "int64":
        return build_array("int64", rng.integers(-2**62, 2**62, n, dtype=np.int64), valid)
    if kind == "int64_dups":
        return build_array("int64", rng.integers(0, 40, n, dtype=np.int64), valid)
    if kind == "uint32":
        return build_array("uint32", rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32), valid)
    if kind == "int16":
        return build_array("int16", rng.integers(-2**15, 2**15, n).astype(np.int16), valid)
    if kind == "float64":
        v = rng.standard_normal(n)
        v[rng.random(n) < 0.05] = np.nan
        v[rng.random(n) < 0.05] = -0.0
        v[rng.random(n) < 0.02] = np.inf
        return build_array("double", v, valid)
    if kind == "float32":
        v = rng.standard_normal(n).astype(np.float32)
        v[rng.random(n) < 0.05] = np.float32("nan")
        v[rng.random(n) < 0.01] = -np.float32("nan")
        return build_array("float", v, valid)
    raise AssertionError(kind)


@pytest.mark.parametrize("kind", ["int64", "int64_dups", "uint32", "int16", "float64", "float32"])
@pytest.mark.parametrize("largest", [False, True])
@pytest.mark.parametrize("placement", PLACEMENTS)
def test_top_k_is_the_argsort_prefix(am, kind, largest, placement):
    rng = np.random.default_rng(zlib.crc32(f"{kind}/{largest}/{placement}".encode()))
    n = 1_000_003
    col = am.MetalArray.from_arrow(column(rng, kind, n))
    for order in (ORDERS if kind.startswith("float") else ("ieee",)):
        full = ids(col.argsort(largest, placement, order))
        for k in (1, 7, 1000, 4095, 4096, 65_537, 200_000, 230_000, 260_000, n - 1, n, n + 5):
            got = ids(col.top_k(k, largest, placement, order))
            assert np.array_equal(got, full[:k]), (kind, largest, placement, order, k)


def test_constant_all_null_and_category_heavy(am):
    n = 300_000
    cases = [pa.array(np.full(n, 7, dtype=np.int64)),
             pa.array([None] * n, type=pa.int32()),
             pa.array(np.where(np.arange(n) % 3 == 0, np.nan, 1.5)),
             pa.array(np.arange(n, dtype=np.float64), mask=np.arange(n) % 2 == 0)]
    for arr in cases:
        col = am.MetalArray.from_arrow(arr)
        for placement in PLACEMENTS:
            for largest in (False, True):
                full = ids(col.argsort(largest, placement))
                for k in (0, 1, 10, 50_000, 149_999, 150_000, 150_001, n):
                    assert np.array_equal(ids(col.top_k(k, largest, placement)), full[:k]), (arr.type, placement, k)


def test_top_k_at_the_order_by_scale(am):
    # 50M int64 keys as the ORDER BY benchmark's key column: LIMIT-sized answers from the selection.
    rng = np.random.default_rng(20260906 + 2)
    n = 50_000_000
    key = rng.integers(0, 2**40, n, dtype=np.int64)
    valid = rng.random(n) >= 0.10
    col = am.MetalArray.from_arrow(pa.array(key, mask=~valid))
    vi = np.flatnonzero(valid)
    order = vi[np.argsort(key[vi], kind="stable")]
    for k in (10, 1000, 1_000_000):
        assert np.array_equal(ids(col.top_k(k, False)), order[:k])
