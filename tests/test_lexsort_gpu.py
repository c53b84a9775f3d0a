"""Multi-key sort on the GPU: pyarrow's sort_indices (golden and live), per-key options against the
oracle, and the paths where a lower key's null rows fold into its key range or need a category pass."""
import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def test_golden_lexsort(am):
    g = golden()
    for c in g.cases:
        if c["kind"] != "lexsort":
            continue
        arrays = [am.MetalArray.from_arrow(g.array(n, t)) for n, t in zip(c["arrays"], c["types"])]
        got = ids(am.lexsort_indices(arrays, c["descending"], c["null_placement"]))
        assert np.array_equal(got, g[c["expect"]]), c


def _col(rng, kind, n, nf):
    mask = rng.random(n) < nf if nf else None
    if kind == "i64_full":
        return pa.array(rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64, endpoint=True), mask=mask)
    if kind == "i64_narrow":
        return pa.array(rng.integers(0, 50, n), mask=mask)
    if kind == "u64_low":
        return pa.array(rng.integers(0, 3, n).astype(np.uint64), mask=mask)
    if kind == "i32":
        return pa.array(rng.integers(-5, 5, n).astype(np.int32), mask=mask)
    if kind == "f64":
        v = rng.normal(0, 10, n).round(1)
        v[rng.random(n) < 0.05] = np.nan
        v[rng.random(n) < 0.05] = -0.0
        return pa.array(v, mask=mask)
    if kind == "f32":
        v = rng.integers(-3, 3, n).astype(np.float32)
        v[rng.random(n) < 0.1] = np.nan
        return pa.array(v, mask=mask)
    if kind == "bool":
        return pa.array(rng.random(n) < 0.5, mask=mask)
    raise ValueError(kind)


@pytest.mark.parametrize("kinds", [("i32", "f64"), ("f64", "i64_full"), ("i64_narrow", "i64_full", "f32"),
                                   ("bool", "u64_low", "i64_narrow"), ("f32", "f32"), ("i64_full", "i64_full")])
@pytest.mark.parametrize("n", [1, 4097, 100_003])
def test_per_key_options_against_oracle(am, oracle, kinds, n):
    rng = np.random.default_rng(n + len(kinds))
    for trial in range(4):
        cols = [_col(rng, k, n, [0.0, 0.1, 0.5][trial % 3]) for k in kinds]
        desc = [bool(rng.random() < 0.5) for _ in kinds]
        place = [("at_end", "at_start")[int(rng.random() < 0.5)] for _ in kinds]
        fo = [("ieee", "total", "nan_largest")[int(rng.integers(0, 3))] for _ in kinds]
        got = ids(am.lexsort_indices([am.MetalArray.from_arrow(c) for c in cols], desc, place, fo))
        want = oracle.lexsort(cols, desc, place, fo)
        assert np.array_equal(got, want), (kinds, desc, place, fo)
        if n <= 4097:
            assert np.array_equal(got, oracle.np_lexsort(cols, desc, place, fo))


def test_lower_key_without_room_takes_category_pass(am, oracle):
    # The lower key uses the whole int64 range and has nulls: no spare key for its null rows.
    rng = np.random.default_rng(8)
    n = 200_000
    hi = pa.array(rng.integers(0, 4, n))
    v = rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64, endpoint=True)
    v[:2] = [-2**63, 2**63 - 1]
    lo = pa.array(v, mask=rng.random(n) < 0.2)
    for place in ("at_end", "at_start"):
        got = ids(am.lexsort_indices([hi, lo], [False, True], place))
        table = pa.table({"a": hi, "b": lo})
        want = pc.sort_indices(table, [("a", "ascending"), ("b", "descending")], null_placement=place).to_numpy()
        assert np.array_equal(got, want), place


def test_config_shaped_multikey(am, oracle):
    # Two keys as in the 50M multi-key workload, at 2M rows: int32 from 200 distinct values (Zipf 1.1)
    # descending, float64 N(0, 1e6) ascending with -0.0 / +0.0 / +-inf / NaN and 5% nulls.
    rng = np.random.default_rng(20260909)
    n = 2_000_000
    distinct = rng.choice(np.arange(-2**31, 2**31 - 1, dtype=np.int64), 200, replace=False).astype(np.int32)
    p = np.arange(1, 201, dtype=np.float64) ** -1.1
    key1 = distinct[rng.choice(200, n, p=p / p.sum())]
    key2 = rng.normal(0, 1e6, n)
    pos = rng.permutation(n)
    for j, val in enumerate([-0.0, 0.0, np.inf, -np.inf]):
        key2[pos[j * n // 200:(j + 1) * n // 200]] = val
    key2[pos[4 * n // 200:6 * n // 200]] = np.nan
    k2 = pa.array(key2, mask=rng.random(n) < 0.05)
    k1 = pa.array(key1)
    got = ids(am.lexsort_indices([k1, k2], [True, False]))
    want = pc.sort_indices(pa.table({"a": k1, "b": k2}), [("a", "descending"), ("b", "ascending")]).to_numpy()
    assert np.array_equal(got, want)
