"""The multi-GPU path of bench.py (replicas, one process per GPU) on CPU: two gloo
ranks with different timings combine to the slowest rank's times and the whole-job
rate counts both ranks' work; with one rank nothing is exchanged."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as tmp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        mine = [10.0 + rank, 20.0 - rank, 5.0 * (rank + 1)]
        got = bench.max_over_ranks(mine, world, "cpu")
        out[rank] = (got, bench.job_rate(64, world, got[0]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_replicas_combine_to_the_slowest_rank():
    world, port = 2, _free_port()
    mgr = tmp.get_context("spawn").Manager()
    out = mgr.dict()
    tmp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        got, rate = out[r]
        assert got == [11.0, 20.0, 10.0]
        assert rate == pytest.approx(128 / 0.011)


def test_single_rank_is_local():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5], 1, "cpu") == [1.5, 2.5]
    assert bench.job_rate(64, 1, 2.0) == pytest.approx(32000.0)


def test_sub_batches_keep_every_pairs_rotation_step():
    """Splitting the 64-pair step into sub-batches keeps the work of the whole batch:
    per rotation step, the sub-batches' runs count exactly the pairs that take it, and
    each sub-batch's runs tile its pairs."""
    import bench
    import ckks_step
    steps, pairs = len(bench.STEPS_K), bench.DEFAULT_PAIRS
    whole = {g: cnt for g, _, cnt in ckks_step.rotation_runs(0, pairs, steps)}
    assert sum(whole.values()) == pairs
    for count in (1, 2, 4, 8):
        pc = pairs // count
        got = {}
        for c in range(count):
            runs = ckks_step.rotation_runs(c * pc, pc, steps)
            assert [r[1] for r in runs] == [sum(r[2] for r in runs[:k]) for k in range(len(runs))]
            assert sum(r[2] for r in runs) == pc
            for g, _, cnt in runs:
                got[g] = got.get(g, 0) + cnt
        assert got == whole
        rows = ckks_step.row_groups(pairs, count, steps)
        assert len(rows) == pairs and {g: rows.count(g) for g in set(rows)} == whole
