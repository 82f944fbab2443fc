"""Cell sharding on the GPU, with the shards run one after another on one
device: each shard's context walks its cell range over only the nets its
cells read, exports its accumulator block, the blocks are summed
element-wise by type (as the ranks' all-reduces would), and the sum is
imported into one shard's context. Its results must equal the whole design
walked by one context: per-cycle waveforms bit for bit (integer bins), per
cell bit for bit, counts equal to the oracle's."""
import numpy as np
import pytest

from tests.parity import compare

pytestmark = pytest.mark.gpu


def _sum_blocks(blocks, segments):
    import torch
    out = blocks[0].clone()
    dt = {"float64": torch.float64, "int64": torch.int64, "int32": torch.int32}
    for name, off, n, d in segments:
        nb = n * np.dtype(d).itemsize
        acc = out[off:off + nb].view(dt[d])
        for b in blocks[1:]:
            acc += b[off:off + nb].view(dt[d])
    return out


@pytest.mark.parametrize("n_shard", [2, 3])
def test_shards_sum_to_whole_design(n_shard):
    from gtpower_b200 import B200Power, shard, synth
    from oracle import oracle as orc
    d, info = synth.flat_design(synth.FlatSpec(n_cell=4000, n_cycle=120, seed=61))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=0.1), seed=62).full()
    shards = shard.partition_cells(d, n_shard, np.diff(ev.net_off))
    engines, blocks = [], []
    try:
        for r in range(n_shard):
            e = shard.ShardedPower(d, r, n_shard, shards=shards, device=0, collect_counts=True)
            engines.append(e)
            e.read_power_activities(shard.shard_events(d, ev, *shards[r]))
            blocks.append(e.export_block())
        total = _sum_blocks(blocks, engines[0].segments)
        engines[0].import_block(total)
        got = engines[0].engine.fetch(counts=True)
    finally:
        for e in engines:
            e.close()
    with B200Power(d, device=0, collect_counts=True) as whole:
        whole.read_power_activities(ev)
        ref = whole.fetch(counts=True)
    assert np.array_equal(got.cycle5, ref.cycle5)
    assert np.array_equal(got.cell5, ref.cell5)
    np.testing.assert_allclose(got.totals, ref.totals, rtol=1e-12)
    compare(got, orc.run(d, ev))


def test_single_shard_is_the_whole_design():
    """One rank (world 1): the reduce is the identity."""
    from gtpower_b200 import B200Power, shard, synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=1000, n_cycle=50, seed=63))
    ev = synth.Trace(d, info, synth.TraceSpec(), seed=64).full()
    with shard.ShardedPower(d, 0, 1, device=0) as e:
        e.read_power_activities(ev)
        got = e.fetch()
        again = e.fetch()          # fetched twice: reduced once
    with B200Power(d, device=0) as whole:
        whole.read_power_activities(ev)
        ref = whole.fetch()
    assert np.array_equal(got.cycle5, ref.cycle5) and np.array_equal(again.cycle5, ref.cycle5)
    assert np.array_equal(got.cell5, ref.cell5)
