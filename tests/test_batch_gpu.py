"""Batched evaluation on the GPU: designs of uneven size and length walked
window by window in persistent launches equal the oracle per design; corner
results folded from one walk equal the oracle on the scaled library; the
captured launch sequence is replayed while the window buffers stay."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(800, 40), (3000, 150), (1500, 75), (6000, 60), (400, 110)]


def _workload(window):
    from gtpower_b200 import synth
    designs, streams = [], []
    for i, (nc, ncyc) in enumerate(SIZES):
        d, info = synth.flat_design(synth.FlatSpec(n_cell=nc, n_cycle=ncyc, seed=40 + i))
        spec = synth.TraceSpec(glitch_p=0.1)
        designs.append((d, info, spec, 50 + i))
        streams.append(synth.DeviceStream(synth.Trace(d, info, spec, seed=50 + i), window))
    return designs, streams


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_oracle_and_folds_corners(use_graph):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from gtpower_b200 import B200Power, batch, synth
    from oracle import oracle as orc
    from tests.parity import compare
    designs, streams = _workload(16)
    engines = [B200Power(d, collect_counts=True, cycles_per_tile=8, gates_per_block=256)
               for d, _, _, _ in designs]
    bufs = [None] * len(engines)
    with batch.BatchPower(engines, use_graph=use_graph) as bp:
        while True:
            wins = [s.next(out=bufs[i]) for i, s in enumerate(streams)]
            if all(w is None for w in wins):
                break
            bufs = [w if w is not None else bufs[i] for i, w in enumerate(wins)]
            torch.cuda.synchronize()
            bp.push(wins)
            bp.sync()
        st = bp.stats()
    assert st["launches"] >= 1
    if use_graph:
        assert st["graph_replays"] >= 1
    for (d, info, spec, seed), eng in zip(designs, engines):
        full = synth.Trace(d, info, spec, seed=seed).full()
        res = eng.fetch(counts=True)
        compare(res, orc.run(d, full))
        for ls, is_ in ((0.8, 0.8), (1.3, 1.3), (0.8, 1.3)):
            dc = dataclasses.replace(d, lib=d.lib.scaled(ls, is_))
            compare(batch.fold_corner(res, ls, is_), orc.run(dc, full), check_counts=False)
        eng.close()


def test_batch_equals_one_design_at_a_time():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from gtpower_b200 import B200Power, batch
    designs, streams = _workload(1000)  # one window per design
    wins = [s.next() for s in streams]
    torch.cuda.synchronize()
    a = [B200Power(d) for d, _, _, _ in designs]
    b = [B200Power(d) for d, _, _, _ in designs]
    with batch.BatchPower(a) as bp:
        bp.push(wins)
        bp.sync()
    # the flat designs' one clock net is periodic: the persistent walk took it as runs
    assert all(x.clock_run_nets() == (1, 1) for x in a)
    batch.run_sequential(b, wins)
    for x, y in zip(a, b):
        rx, ry = x.fetch(), y.fetch()
        assert np.allclose(rx.cell5, ry.cell5, rtol=1e-6, atol=0)
        assert np.allclose(rx.cycle5, ry.cycle5, rtol=1e-6, atol=1e-30)
        assert np.allclose(rx.totals, ry.totals, rtol=1e-12)
        x.close()
        y.close()
