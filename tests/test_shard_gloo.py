"""Cell sharding of one design across ranks, on the CPU as two and three
gloo ranks: each rank takes the contiguous cell range partition_cells gives
it and only the events of the nets those cells read (shard_events), walks
it with the FP64 oracle, and the ranks sum their blocks with
all_reduce_block, the collectives the GPU ranks use. The merged result must
equal the oracle over the whole design: integer counts bit for bit, per-cell
values bit for bit (each cell lives on one rank), per-cycle sums within
FP64 rounding."""
import datetime
import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=1500, n_cycle=60, seed=51))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=0.1), seed=52).full()
    return d, ev


def _block(res, n_cell, n_period):
    """The oracle's results in the segment order of the engine's accumulator
    block (per-cycle powers in FP64 in place of the fixed-point bins)."""
    import torch
    parts = [res.cell5.astype(np.float64).ravel(), res.cycle5.astype(np.float64).ravel(),
             np.concatenate([res.cycle_events, res.cycle_glitches]).astype(np.int64),
             np.concatenate([res.cell_events, res.cell_glitches, res.cell_half_toggles,
                             res.cell_related]).astype(np.int32)]
    segs, off = [], 0
    for name, a in zip(("cell", "cycle", "cycle_counts", "cell_counts"), parts):
        segs.append((name, off, a.size, str(a.dtype)))
        off += a.nbytes
    blk = torch.from_numpy(np.concatenate([a.view(np.uint8) for a in parts]).copy())
    return blk, segs


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from gtpower_b200 import shard
    from oracle import oracle as orc
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        d, ev = _case()
        shards = shard.partition_cells(d, world, np.diff(ev.net_off))
        b, e = shards[rank]
        sev = shard.shard_events(d, ev, b, e)
        r = orc.run(d, sev, cells=np.arange(b, e, dtype=np.int32))
        blk, segs = _block(r, d.n_cell, d.n_period)
        shard.all_reduce_block(blk, segs, dist)
        q.put((rank, shards, blk.numpy().copy(), sev.n_event))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_ranks_sum_to_the_whole_design(world):
    mp = pytest.importorskip("torch.multiprocessing")
    from oracle import oracle as orc
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = mp.spawn(_rank_main, args=(world, _free_port(), q), nprocs=world, join=False)
    got = {}
    for _ in range(world):  # drain the queue before joining: the blocks exceed a pipe's buffer
        rank, shards, blk, n_ev = q.get()
        got[rank] = (shards, blk, n_ev)
    while not procs.join():
        pass
    d, ev = _case()
    ref = orc.run(d, ev)
    ref_blk, segs = _block(ref, d.n_cell, d.n_period)
    ref_blk = ref_blk.numpy()
    shards = got[0][0]
    # the ranges cover every cell once, and each rank got fewer events
    assert shards[0][0] == 0 and shards[-1][1] == d.n_cell
    assert all(shards[i][1] == shards[i + 1][0] for i in range(world - 1))
    assert all(got[r][2] < ev.n_event for r in range(world))
    for r in range(world):
        blk = got[r][1]
        assert blk.shape == ref_blk.shape
        for name, off, n, dt in segs:
            a = blk[off:off + n * np.dtype(dt).itemsize].view(dt)
            b = ref_blk[off:off + n * np.dtype(dt).itemsize].view(dt)
            if name == "cycle":
                np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())
            else:
                assert np.array_equal(a, b), name


def test_partition_balances_work():
    from gtpower_b200 import shard
    d, ev = _case()
    cnt = np.diff(ev.net_off)
    sh = shard.partition_cells(d, 4, cnt)
    w = shard._cell_pin_events(d, cnt)
    per = [int(w[b:e].sum()) for b, e in sh]
    assert max(per) <= 1.1 * (sum(per) / 4) + int(w.max())
    assert shard.partition_cells(d, 1) == [(0, d.n_cell)]
