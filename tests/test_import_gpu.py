"""Imports from pinned host memory: the copies run asynchronously on the importing thread's copy stream
and the producer's buffers are released once they are done; every use of the array waits for them."""
import numpy as np
import pyarrow as pa
import pytest

pytestmark = pytest.mark.gpu


def pinned(torch, arr, keep):
    bufs = []
    for b in arr.buffers():
        if b is None:
            bufs.append(None)
            continue
        t = torch.empty(b.size, dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = np.frombuffer(b, dtype=np.uint8)
        keep.append(t)
        bufs.append(pa.py_buffer(t.numpy()))
    return pa.Array.from_buffers(arr.type, len(arr), bufs, null_count=arr.null_count, offset=arr.offset)


def test_pinned_import_round_trips_and_sorts(am):
    import torch
    rng = np.random.default_rng(21)
    keep = []
    n = 3_000_000
    src = {"k": pa.array(rng.integers(-2**40, 2**40, n), mask=rng.random(n) < 0.1),
           "f": pa.array(rng.standard_normal(n)),
           "i": pa.array(rng.integers(-100, 100, n).astype(np.int32))}
    host = {k: pinned(torch, v, keep) for k, v in src.items()}
    for _ in range(3):
        dev = {k: am.MetalArray.from_arrow(v) for k, v in host.items()}
        for k in src:
            assert dev[k].to_arrow().equals(src[k]), k
        idx = dev["k"].argsort().to_arrow().to_numpy()
        want = np.argsort(np.where(np.asarray(src["k"].is_valid()), src["k"].fill_null(0).to_numpy(), 2**62),
                          kind="stable")
        assert np.array_equal(idx, want)
        out = am.run_plan({"op": "sort", "by": [["k", False]], "input": {"op": "scan", "source": "t"}},
                          [am.PlanSource("t", dev)])
        assert out["f"].to_arrow().equals(src["f"].take(pa.array(idx)))


def test_pinned_import_of_a_sliced_array(am):
    import torch
    keep = []
    base = pa.array(np.arange(100_000, dtype=np.int64), mask=np.arange(100_000) % 7 == 0)
    host = pinned(torch, base, keep)
    for off in (0, 8, 13):
        sl = host.slice(off, 50_000)
        got = am.MetalArray.from_arrow(sl).to_arrow()
        assert got.equals(base.slice(off, 50_000)), off
