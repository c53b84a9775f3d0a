"""The two-level single-key sort (two passes on the top digits, then shared-memory sorts of the
buckets, or the remaining passes when a bucket is too large) at the sizes that take it: at least 2^25
value rows of one 8-byte key. Every permutation must equal the oracle's stable argsort, whichever path
the device picks: uniform keys (local sorts of every shape, chosen by bucket size), a heavily repeated
key (the fallback passes), floats with NaN and -0.0, full-range keys (six local digits), both
directions and null placements, and the ORDER BY's rebuilt key column."""
import numpy as np
import pyarrow as pa
import pytest

pytestmark = pytest.mark.gpu

N = 40_000_000          # 10% nulls still leave more than 2^25 value rows


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def check(am, oracle, arr, desc=False, placement="at_end", float_order="ieee"):
    got = ids(am.MetalArray.from_arrow(arr).argsort(desc, placement, float_order))
    want = oracle.np_argsort(arr, desc, placement, float_order)
    assert np.array_equal(got, want), (desc, placement, float_order)


@pytest.mark.parametrize("desc,placement", [(False, "at_end"), (True, "at_start")])
def test_uniform_40_bit_keys(am, oracle, desc, placement):
    rng = np.random.default_rng(11)
    arr = pa.array(rng.integers(0, 2**40, N, dtype=np.int64), mask=rng.random(N) < 0.10)
    check(am, oracle, arr, desc, placement)


@pytest.mark.parametrize("top_bits", [15, 14])
def test_bucket_sizes_for_the_larger_shapes(am, oracle, top_bits):
    # 2^15 and 2^14 distinct top-16 values: buckets of ~1,100 and ~2,200 rows.
    rng = np.random.default_rng(12 + top_bits)
    top = rng.integers(0, 2**top_bits, N, dtype=np.int64) << 24
    arr = pa.array(top | rng.integers(0, 2**24, N, dtype=np.int64))
    check(am, oracle, arr)


def test_repeated_key_takes_the_fallback_passes(am, oracle):
    rng = np.random.default_rng(13)
    key = rng.integers(0, 2**40, N, dtype=np.int64)
    key[rng.random(N) < 0.3] = 123_456_789_012                  # one bucket of ~12M rows
    arr = pa.array(key, mask=rng.random(N) < 0.05)
    check(am, oracle, arr)
    check(am, oracle, arr, True, "at_start")


def test_full_range_keys_and_three_digit_keys(am, oracle):
    rng = np.random.default_rng(14)
    check(am, oracle, pa.array(rng.integers(-2**63, 2**63 - 1, N, dtype=np.int64)))
    check(am, oracle, pa.array(rng.integers(0, 2**24, N, dtype=np.int64).astype(np.uint64)), True)


def test_floats_with_nan_and_signed_zero(am, oracle):
    rng = np.random.default_rng(15)
    v = rng.standard_normal(N)
    v[rng.random(N) < 0.02] = np.nan
    v[rng.random(N) < 0.02] = -0.0
    v[rng.random(N) < 0.02] = 0.0
    arr = pa.array(v, mask=rng.random(N) < 0.03)
    for placement in ("at_end", "at_start"):
        check(am, oracle, arr, False, placement)
    check(am, oracle, arr, True, "at_end", "total")


def test_order_by_rebuilds_the_key_column(am):
    rng = np.random.default_rng(16)
    key = rng.integers(-2**50, 2**50, N, dtype=np.int64)
    valid = rng.random(N) >= 0.1
    payload = rng.standard_normal(N)
    src = am.PlanSource("t", {"k": pa.array(key, mask=~valid), "p": pa.array(payload)})
    out = am.run_plan({"op": "sort", "by": [["k", True, {"nulls": "first"}]], "input": {"op": "scan", "source": "t"}},
                      [src])
    vi = np.flatnonzero(valid)
    order = vi[np.argsort(-key[vi], kind="stable")]
    nulls = np.flatnonzero(~valid)
    k = out["k"].to_arrow()
    nn = len(nulls)
    assert k.null_count == nn
    assert np.array_equal(np.frombuffer(k.buffers()[1], dtype=np.int64)[nn:N], key[order])
    assert np.array_equal(out["p"].to_arrow().to_numpy(), payload[np.concatenate([nulls, order])])
