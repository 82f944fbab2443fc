"""The multi-process path of bench.py, run on the CPU as two gloo ranks: the
timing reduction keeps the slowest rank's time, every rank evaluates its own
trace of the same design (weak scaling, no data-path collective), and the
reference arm does its work on rank 0 only."""
import datetime
import os
import socket
import types

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        assert bench.dist_env() == (rank, world, rank)
        slowest = bench.max_over_ranks(dist, [1.0 + rank, 10.0 - rank, 3.0], "cpu")
        design, _, trace = bench.workload(types.SimpleNamespace(cells=300, cycles=20), rank)
        ev = trace.full()
        mine = torch.tensor([float(design.n_cell), float(design.n_pin), float(ev.n_event),
                             float(ev.time.sum() % 1_000_003)], dtype=torch.float64)
        all_ranks = [torch.zeros(4, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(all_ranks, mine)
        if rank != 0:
            assert bench.run_reference(types.SimpleNamespace(), rank, world) is None
        q.put((rank, slowest, [t.tolist() for t in all_ranks]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_times_and_walk_their_own_traces():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.spawn(_rank_main, args=(2, _free_port(), q), nprocs=2, join=True)
    res = {}
    for _ in range(2):
        rank, slowest, all_ranks = q.get()
        res[rank] = (slowest, all_ranks)
    assert sorted(res) == [0, 1]
    for rank in (0, 1):
        slowest, (r0, r1) = res[rank]
        assert slowest == [2.0, 10.0, 3.0]  # each value's maximum over the two ranks
        assert r0[:2] == r1[:2]             # the same design on both ranks
        assert r0[2:] != r1[2:]             # each rank its own trace
    assert res[0][1] == res[1][1]


def test_max_over_ranks_without_a_process_group():
    import bench
    assert bench.max_over_ranks(None, [3, 1.5], "cpu") == [3.0, 1.5]


def test_metric_names_the_workload_size():
    import bench
    assert bench.metric_name(200_000, 10_000) == \
        "net events/s (time-based power walk, flat synthetic 200k cells x 10k cycles)"
    assert bench.metric_name(2000, 50) == "net events/s (time-based power walk, flat synthetic 2k cells x 50 cycles)"


def test_reference_arm_line_names_the_engine_workload(capsys):
    """The reference arm's line carries the same metric and config.workload
    as the engine's line (both built by bench.metric_name / workload_name),
    times every cell each timed step, and declares zero copies."""
    import json
    import bench
    args = types.SimpleNamespace(cells=400, cycles=30, steps=1, warmup=1)
    bench.run_reference(args, 0, 1)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.metric_name(400, 30)
    assert line["config"]["workload"] == bench.workload_name(args)
    assert "all 400 cells" in line["cpu_baseline"]["sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
