"""The sort server (am_server_*): each request's result in a mix of concurrent, batched requests equals
the same request run alone through am_plan_run; admission keeps the footprint in flight under the cap;
bad requests fail at submission with the library's error convention."""
import json

import numpy as np
import pyarrow as pa
import pytest

from conftest import build_array

pytestmark = pytest.mark.gpu

N = 600_000


def table(am, seed=5):
    return table_and_columns(am, seed)[0]


def table_and_columns(am, seed=5):
    rng = np.random.default_rng(seed)
    k64 = build_array("int64", rng.integers(-2**40, 2**40, N, dtype=np.int64), rng.random(N) > 0.05)
    fv = rng.standard_normal(N)
    fv[rng.random(N) < 0.02] = np.nan
    fv[rng.random(N) < 0.01] = -0.0
    kf = build_array("double", fv, rng.random(N) > 0.03)
    k32 = pa.array(rng.integers(0, 300, N).astype(np.int32))
    p1 = pa.array(rng.standard_normal(N))
    p2 = pa.array(rng.integers(-2**31, 2**31 - 1, N, dtype=np.int32, endpoint=True))
    cols = {"k64": k64, "kf": kf, "k32": k32, "p1": p1, "p2": p2}
    return am.PlanSource("t", {k: am.MetalArray.from_arrow(v) for k, v in cols.items()}), cols


def plan_alone(offset, length, keys, desc, nulls, orders, payload):
    cols = list(keys) + list(payload)
    sel = [[c, f'(col "{c}")'] for c in cols]
    by = [[k, d, {"nulls": "first" if n == "at_start" else "last", "float_order": o}]
          for k, d, n, o in zip(keys, desc, nulls, orders)]
    return json.dumps({"op": "select", "exprs": sel, "input": {"op": "sort", "by": by, "input": {
        "op": "select", "exprs": sel, "input": {"op": "limit", "count": length, "offset": offset,
                                                "input": {"op": "scan", "source": "t"}}}}})


def same(a, b):
    """Equal validity and equal value bits at every valid row."""
    if len(a) != len(b) or a.type != b.type or a.null_count != b.null_count:
        return False
    va = np.asarray(a.is_valid().to_numpy(zero_copy_only=False))
    vb = np.asarray(b.is_valid().to_numpy(zero_copy_only=False))
    if not np.array_equal(va, vb):
        return False
    view = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[a.type.bit_width // 8]
    xa = np.frombuffer(a.buffers()[1], dtype=view)[a.offset:a.offset + len(a)]
    xb = np.frombuffer(b.buffers()[1], dtype=view)[b.offset:b.offset + len(b)]
    return np.array_equal(xa[va], xb[vb])


def random_requests(rng, count):
    reqs = []
    for _ in range(count):
        length = int(min(N, round(10 ** rng.uniform(0, np.log10(N)))))
        offset = int(rng.integers(0, N - length + 1))
        kind = rng.integers(4)
        if kind == 0:
            keys, orders = ["k64"], ["ieee"]
        elif kind == 1:
            keys, orders = ["kf"], [["ieee", "total", "nan_largest"][rng.integers(3)]]
        elif kind == 2:
            keys, orders = ["k32", "k64"], ["ieee", "ieee"]
        else:
            keys, orders = ["k32", "kf"], ["ieee", "total"]
        desc = [bool(rng.integers(2)) for _ in keys]
        nulls = [["at_end", "at_start"][rng.integers(2)] for _ in keys]
        reqs.append((offset, length, keys, desc, nulls, orders, ["p1", "p2"]))
    return reqs


def test_mix_equals_alone(am):
    src = table(am)
    rng = np.random.default_rng(9)
    reqs = random_requests(rng, 80)
    alone = [am.run_plan(plan_alone(*r), [src]) for r in reqs]
    with am.Server(workers=4, hbm_cap_bytes=8 << 30, batch_rows=1 << 17) as srv:
        tickets = [srv.submit(src, o, n, k, p, descending=d, null_placement=nl, float_order=fo)
                   for (o, n, k, d, nl, fo, p) in reqs]
        results = [srv.wait(t) for t in tickets]
        stats = srv.stats()
    assert stats["requests"] == len(reqs)
    assert stats["batches"] > 0 and stats["solo_requests"] > 0
    for r, want, (got, latency) in zip(reqs, alone, results):
        assert latency >= 0
        assert list(got) == list(want), r
        for name in want:
            assert same(got[name].to_arrow(), want[name].to_arrow()), (r, name)


def expected_order(oracle, cols, offset, length, keys, desc, nulls, orders):
    """Row numbers (within the slice) of the request's sort: pyarrow's sort_indices where its options
    can say it (ieee order, one null placement for every key), else the oracle's definition."""
    import pyarrow.compute as pc
    part = {k: cols[k].slice(offset, length) for k in keys}
    if all(o == "ieee" for o in orders) and len(set(nulls)) == 1:
        t = pa.table(part)
        by = [(k, "descending" if d else "ascending") for k, d in zip(keys, desc)]
        return pc.sort_indices(t, sort_keys=by, null_placement=nulls[0]).to_numpy().astype(np.int64)
    return oracle.np_lexsort([part[k] for k in keys], desc, nulls, orders).astype(np.int64)


def test_served_results_match_pyarrow_on_a_sample(am, oracle):
    # A sampled subset of a served mix, checked outside the library: the order against pyarrow's
    # sort_indices (or the oracle where pyarrow has no such order), the columns against pyarrow's take
    # of the source slice through that order.
    src, cols = table_and_columns(am, seed=10)
    rng = np.random.default_rng(12)
    reqs = random_requests(rng, 60)
    with am.Server(workers=4, hbm_cap_bytes=8 << 30, batch_rows=1 << 17) as srv:
        tickets = [srv.submit(src, o, n, k, p, descending=d, null_placement=nl, float_order=fo)
                   for (o, n, k, d, nl, fo, p) in reqs]
        results = [srv.wait(t)[0] for t in tickets]
    sample = rng.choice(len(reqs), 20, replace=False)
    for i in sample:
        offset, length, keys, desc, nulls, orders, payload = reqs[i]
        order = pa.array(expected_order(oracle, cols, offset, length, keys, desc, nulls, orders))
        got = results[i]
        assert list(got) == list(keys) + list(payload), reqs[i]
        for name in got:
            want = cols[name].slice(offset, length).take(order)
            assert same(got[name].to_arrow(), want), (reqs[i], name)


def test_admission_keeps_footprint_under_cap(am):
    src = table(am, seed=6)
    # Each 200,000-row request needs about 200,000 x 45 B + 1 MiB (~10 MB); a 25 MB cap admits two.
    cap = 25_000_000
    with am.Server(workers=4, hbm_cap_bytes=cap, batch_rows=0) as srv:
        tickets = [srv.submit(src, 1000 * i, 200_000, ["k64"], ["p1", "p2"]) for i in range(12)]
        for t in tickets:
            srv.wait(t)
        stats = srv.stats()
    assert stats["requests"] == 12
    assert 0 < stats["peak_in_flight_bytes"] <= cap
    assert stats["in_flight_bytes"] == 0 and stats["queued"] == 0


def test_request_larger_than_the_cap_runs_alone(am):
    src = table(am, seed=7)
    with am.Server(workers=2, hbm_cap_bytes=1_000_000, batch_rows=0) as srv:
        got, _ = srv.wait(srv.submit(src, 0, N, ["k64"], ["p2"]))
    want = am.run_plan(plan_alone(0, N, ["k64"], [False], ["at_end"], ["ieee"], ["p2"]), [src])
    for name in want:
        assert same(got[name].to_arrow(), want[name].to_arrow())


def test_bad_requests_fail_at_submission(am):
    src = table(am, seed=8)
    with am.Server(workers=1) as srv:
        with pytest.raises(am.ArrowMetalError, match="unknown column"):
            srv.submit(src, 0, 10, ["nope"], ["p1"])
        with pytest.raises(am.ArrowMetalError, match="outside the table"):
            srv.submit(src, N - 5, 10, ["k64"], ["p1"])
        got, _ = srv.wait(srv.submit(src, 10, 0, ["k64"], ["p1"]))
        assert all(len(v) == 0 for v in got.values())


def test_shared_sorts_equal_each_request_alone(am, oracle):
    # Queued requests of one table, key and options over overlapping slices share one sort of the rows
    # they cover; each result must still equal the request alone and pyarrow's order of its slice.
    src, cols = table_and_columns(am, seed=13)
    rng = np.random.default_rng(14)
    kinds = [(["k64"], [False], ["at_end"], ["ieee"]), (["kf"], [True], ["at_start"], ["total"]),
             (["k32", "k64"], [True, False], ["at_end", "at_start"], ["ieee", "ieee"])]
    reqs = []
    for i in range(48):
        keys, desc, nulls, orders = kinds[i % 3]
        length = int(rng.integers(N // 8, N // 2))
        offset = int(rng.integers(0, N - length + 1))
        reqs.append((offset, length, keys, desc, nulls, orders, ["p1", "p2"]))
    alone = [am.run_plan(plan_alone(*r), [src]) for r in reqs]
    with am.Server(workers=2, hbm_cap_bytes=8 << 30, batch_rows=0) as srv:
        tickets = [srv.submit(src, o, n, k, p, descending=d, null_placement=nl, float_order=fo)
                   for (o, n, k, d, nl, fo, p) in reqs]
        results = [srv.wait(t)[0] for t in tickets]
        stats = srv.stats()
    assert stats["requests"] == len(reqs) and stats["shared_sorts"] > 0 and stats["shared_requests"] > 2
    for r, want, got in zip(reqs, alone, results):
        assert list(got) == list(want), r
        for name in want:
            assert same(got[name].to_arrow(), want[name].to_arrow()), (r, name)
    for i in range(0, len(reqs), 5):
        offset, length, keys, desc, nulls, orders, payload = reqs[i]
        order = pa.array(expected_order(oracle, cols, offset, length, keys, desc, nulls, orders))
        for name in results[i]:
            assert same(results[i][name].to_arrow(), cols[name].slice(offset, length).take(order)), (reqs[i], name)


def test_shared_sorts_mix_compacted_and_gathered_requests(am, oracle):
    # Requests covering at least an eighth of the shared rows get their columns by compaction of the
    # covered rows' columns in the shared order, shorter ones by a take of their own; a payload column
    # may hold nulls. Every result must equal the request alone.
    src, cols = table_and_columns(am, seed=21)
    rng = np.random.default_rng(22)
    reqs = []
    for i in range(40):
        length = int(rng.integers(N // 6, N // 2)) if i % 2 else int(rng.integers(1, N // 40))
        offset = int(rng.integers(0, N - length + 1))
        payload = ["p1", "p2"] if i % 3 else ["p2", "kf"]
        reqs.append((offset, length, ["k64"], [bool(i % 4 == 1)], ["at_start" if i % 5 else "at_end"],
                     ["ieee"], payload))
    alone = [am.run_plan(plan_alone(*r), [src]) for r in reqs]
    with am.Server(workers=1, hbm_cap_bytes=8 << 30, batch_rows=0) as srv:
        tickets = [srv.submit(src, o, n, k, p, descending=d, null_placement=nl, float_order=fo)
                   for (o, n, k, d, nl, fo, p) in reqs]
        results = [srv.wait(t)[0] for t in tickets]
        stats = srv.stats()
    assert stats["shared_sorts"] > 0
    for r, want, got in zip(reqs, alone, results):
        assert list(got) == list(want), r
        for name in want:
            assert same(got[name].to_arrow(), want[name].to_arrow()), (r, name)
    offset, length, keys, desc, nulls, orders, payload = reqs[1]
    order = pa.array(expected_order(oracle, cols, offset, length, keys, desc, nulls, orders))
    for name in results[1]:
        assert same(results[1][name].to_arrow(), cols[name].slice(offset, length).take(order)), name


def test_shared_sorts_can_be_turned_off(am, monkeypatch):
    src = table(am, seed=15)
    monkeypatch.setenv("ARROWMETAL_SERVER_SHARED", "0")
    with am.Server(workers=1, hbm_cap_bytes=8 << 30, batch_rows=0) as srv:
        ts = [srv.submit(src, 1000 * i, N // 2, ["k64"], ["p1"]) for i in range(6)]
        for t in ts:
            srv.wait(t)
        assert srv.stats()["shared_sorts"] == 0
