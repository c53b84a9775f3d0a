"""Multi-GPU runs are independent replicas: each rank sorts its own table, and the benchmark reports the
whole job's rows/s over the slowest rank's time. These tests run that host logic as two `gloo` ranks on
the CPU (no GPU, no collective on the data path)."""
import json
import os
import socket
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out_dir):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(times[rank], dist, "cpu")
        rate = bench.whole_job_rate(1_000_000, world, ms)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"ms": ms, "rate": rate}, f)


def test_two_replicas_report_the_slowest_rank(tmp_path):
    import torch.multiprocessing as mp
    times = [4.0, 5.0]
    mp.start_processes(_rank_main, args=(2, _free_port(), times, str(tmp_path)), nprocs=2, start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for g in got:
        assert g["ms"] == 5.0
        assert g["rate"] == pytest.approx(2 * 1_000_000 / 5e-3)


def test_single_process_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_rate(50_000_000, 1, 5.0) == pytest.approx(1e10)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import bench
    args = types.SimpleNamespace(gpus=2, steps=1, warmup=1)
    assert bench.run_reference_arm(args, rank=1) is None
    assert capsys.readouterr().out == ""
