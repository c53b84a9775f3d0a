"""The plan entry points with the plans the sort's callers send (the DataFusion rule's
select_all(sort(scan)) with limit, the Polars engine's per-key options), against pyarrow."""
import json

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

pytestmark = pytest.mark.gpu


def _table(rng, n):
    return pa.table({"c0": pa.array(rng.integers(0, 2**40, n), mask=rng.random(n) < 0.1),
                     "c1": pa.array(rng.normal(size=n)),
                     "c2": pa.array(rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32))})


def datafusion_plan(keys, fetch=None):
    # datafusion/src/gpu.rs:45-66 and :232-238, verbatim shape.
    by = ",".join(f'["c{c}",{"true" if d else "false"},{{"nulls":"{"first" if nf else "last"}","float_order":"total"}}]'
                  for c, d, nf in keys)
    node = f'{{"op":"sort","by":[{by}],"input":{{"op":"scan","source":"t"}}}}'
    if fetch is not None:
        node = f'{{"op":"limit","count":{fetch},"input":{node}}}'
    exprs = ",".join(f'["c{i}","(col \\"c{i}\\")"]' for i in range(3))
    return f'{{"op":"select","exprs":[{exprs}],"input":{node}}}'


@pytest.mark.parametrize("keys,fetch", [([(0, False, False)], None), ([(0, True, True)], None),
                                        ([(2, False, False), (1, True, False)], None),
                                        ([(0, False, False)], 1000)])
def test_datafusion_shaped_plans(am, keys, fetch):
    rng = np.random.default_rng(len(keys) + (fetch or 0))
    t = _table(rng, 200_001)
    src = am.PlanSource("t", {k: t[k].combine_chunks() for k in t.column_names})
    out = am.run_plan(datafusion_plan(keys, fetch), [src])
    assert list(out) == ["c0", "c1", "c2"]
    place = "at_start" if keys[0][2] else "at_end"
    idx = pc.sort_indices(t, [(f"c{c}", "descending" if d else "ascending") for c, d, _ in keys], null_placement=place)
    if fetch is not None:
        idx = idx[:fetch]
    want = t.take(idx)
    for k in out:
        assert out[k].to_arrow().equals(want[k].combine_chunks()), k


def test_polars_shaped_plan(am, oracle):
    # python/arrowmetal/polars_engine.py:944-998: nulls first unless nulls_last, nan_largest floats.
    rng = np.random.default_rng(5)
    n = 50_000
    v = rng.normal(size=n)
    v[rng.random(n) < 0.05] = np.nan
    a = pa.array(v, mask=rng.random(n) < 0.1)
    b = pa.array(rng.integers(0, 5, n))
    src = am.PlanSource("df", {"a": a, "b": b})
    plan = {"op": "limit", "count": 100, "offset": 10,
            "input": {"op": "sort", "input": {"op": "scan", "source": "df"},
                      "by": [["b", True], ["a", False, {"nulls": "first", "float_order": "nan_largest"}]]}}
    out = am.run_plan(json.dumps(plan), [src])
    idx = oracle.lexsort([b, a], [True, False], ["at_end", "at_start"], ["ieee", "nan_largest"])[10:110]
    assert out["a"].to_arrow().equals(a.take(pa.array(idx)))
    assert out["b"].to_arrow().equals(b.take(pa.array(idx)))
    assert "sort" in am.explain_plan(plan, [src])


def test_plan_errors(am):
    src = am.PlanSource("t", {"x": pa.array([1, 2, 3])})
    with pytest.raises(am.ArrowMetalError, match="unknown sort column"):
        am.run_plan({"op": "sort", "by": [["y", False]], "input": {"op": "scan", "source": "t"}}, [src])
    with pytest.raises(am.ArrowMetalError, match="float_order"):
        am.run_plan({"op": "sort", "by": [["x", False, {"float_order": "x"}]], "input": {"op": "scan", "source": "t"}}, [src])
