"""Failure paths, made on the host or with a wait that runs out -- never a GPU fault: an injected
device-allocation failure, the 2^32 - 1 row refusal (lowered by the test hook, as the reference's
IndexTypeTests.swift:140 lowers Dispatch.maxRowIndex), and a look-back wait given nothing to wait for."""
import numpy as np
import pyarrow as pa
import pytest

pytestmark = pytest.mark.gpu


def test_allocation_failure_is_an_error_and_recoverable(am):
    m = am.MetalArray.from_arrow(pa.array(np.arange(10_000)[::-1].copy()))
    am._lib.am_debug_fail_alloc_after(0)
    try:
        with pytest.raises(am.ArrowMetalError, match="allocation"):
            m.argsort()
    finally:
        am._lib.am_debug_fail_alloc_after(-1)
    assert m.argsort().to_arrow().to_pylist()[:3] == [9999, 9998, 9997]


def test_row_limit_refusal(am):
    m = am.MetalArray.from_arrow(pa.array(np.arange(101)))
    am._lib.am_debug_set_max_row_index(99)
    try:
        with pytest.raises(am.ArrowMetalError, match=r"argsort: row 100 does not fit the UInt32 index type"):
            m.argsort()
        with pytest.raises(am.ArrowMetalError, match="lexsort: row 100"):
            am.lexsort_indices([m, m])
    finally:
        am._lib.am_debug_set_max_row_index(2**32 - 1)
    assert len(m.argsort().to_arrow()) == 101


def test_lookback_wait_runs_out_and_reports(am):
    # int32 keys in [0, 100): one active digit pass over several look-back entries. With the first one
    # skipped, the next one's look-back waits on a status nothing writes, gives up after its time limit
    # and sets the error word.
    rng = np.random.default_rng(1)
    m = am.MetalArray.from_arrow(pa.array(rng.integers(0, 100, 100_000).astype(np.int32)))
    am._lib.am_debug_skip_first_tile(1)
    try:
        with pytest.raises(am.ArrowMetalError, match="look-back"):
            idx = m.argsort()
            am.synchronize()
    finally:
        am._lib.am_debug_skip_first_tile(0)
    got = m.argsort().to_arrow().to_numpy()
    vals = m.to_arrow().to_numpy()
    assert np.array_equal(got, np.argsort(vals, kind="stable"))
