"""One context per host thread: contexts on the same device, driven from
different host threads at the same time (ctypes drops the GIL for the
calls), give the results each gives alone. The ABI keeps no global state
for the walk; each context owns its streams, buffers and accumulators."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(seed):
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=3000, n_cycle=150, seed=seed))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=0.1), seed=seed + 1).full()
    return d, ev


def _run(d, ev, windows=1):
    from gtpower_b200 import B200Power, windows as W
    tpc = d.ticks_per_cycle
    if windows == 1:
        wins = [ev]
    else:
        cuts = np.linspace(0, d.n_period, windows + 1).astype(np.int64) * tpc
        cuts[-1] = np.iinfo(np.int64).max
        wins = [W.make_window(ev, tpc, int(cuts[k]), int(cuts[k + 1])) for k in range(windows)]
    with B200Power(d, device=0, collect_counts=True) as eng:
        for w in wins:
            eng.read_power_activities(w)
        eng.sync()
        return eng.fetch(counts=True)


def test_contexts_in_parallel_host_threads():
    cases = [_case(s) for s in (21, 31, 41, 51)]
    alone = [_run(d, ev, windows=1 + k % 3) for k, (d, ev) in enumerate(cases)]
    out = [None] * len(cases)
    errors = []

    def work(k):
        try:
            d, ev = cases[k]
            for _ in range(3):                 # several rounds each, overlapping the others
                out[k] = _run(d, ev, windows=1 + k % 3)
        except Exception as e:                # reported below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(len(cases))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for k in range(len(cases)):
        assert np.array_equal(out[k].cycle5, alone[k].cycle5), k
        assert np.array_equal(out[k].counts.cell_events, alone[k].counts.cell_events), k
        np.testing.assert_allclose(out[k].cell5, alone[k].cell5, rtol=1e-12, atol=0)
