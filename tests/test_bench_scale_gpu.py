"""Parity at bench scale: the kernel variants the default bench times, on a
flat synthetic design large enough for their fast paths to matter, against
the FP64 oracle.

The default bench configuration (768-cycle tiles, work-sorted cells, clock
pins on exactly periodic nets walked as runs of whole cycles, two-event
buffers per pin) is run three ways on 50k cells x 2k cycles:
  - one device-resident window, as the bench's timed leg pushes it;
  - four host windows growing 1.5x each, as the bench's e2e leg pushes them;
  - with integer counters on (the counting variant of the same walk), whose
    counts must equal the oracle's bit for bit.
"""
import numpy as np
import pytest

from tests.parity import compare

pytestmark = pytest.mark.gpu

N_CELL, N_CYCLE = 50_000, 2_000


@pytest.fixture(scope="module")
def case():
    from gtpower_b200 import synth
    from oracle import oracle as orc
    import os
    d, info = synth.flat_design(synth.FlatSpec(n_cell=N_CELL, n_cycle=N_CYCLE, seed=20261203 + 1))
    ev = synth.Trace(d, info, synth.TraceSpec(), seed=20261203 + 1).full()
    ref = orc.run(d, ev, threads=os.cpu_count() or 1)
    return d, ev, ref


def _ramp_windows(ev, tpc, n_cycle, n_win=4):
    from gtpower_b200 import windows
    sizes = 1.5 ** np.arange(n_win)
    cuts = np.unique(np.concatenate([[0], np.round(np.cumsum(sizes) / sizes.sum() * n_cycle)]).astype(np.int64))
    return [windows.make_window(ev, tpc, int(cuts[k]) * tpc,
                                int(cuts[k + 1]) * tpc if k + 2 < len(cuts) else np.iinfo(np.int64).max)
            for k in range(len(cuts) - 1)]


def test_device_window_default_config(case):
    import torch
    from gtpower_b200 import B200Power
    d, ev, ref = case
    dev = torch.device("cuda", 0)
    d_off = torch.from_numpy(ev.net_off).to(dev)
    d_t = torch.from_numpy(ev.time).to(dev)
    d_v = torch.from_numpy(ev.packed.view(np.int32)).to(dev)
    with B200Power(d, device=0) as eng:
        eng.push_device(ev.n_event, d_off.data_ptr(), d_t.data_ptr(), d_v.data_ptr())
        eng.sync()
        n_clk, n_per = eng.clock_run_nets()
        assert n_clk == 1 and n_per == 1   # the clock net was walked as runs
        res = eng.fetch()
    err = compare(res, ref, check_counts=False)
    assert max(err.values()) <= 1e-5


def test_host_windows_default_config(case):
    from gtpower_b200 import B200Power
    d, ev, ref = case
    wins = _ramp_windows(ev, d.ticks_per_cycle, N_CYCLE)
    with B200Power(d, device=0) as eng:
        for w in wins:
            eng.read_power_activities(w)
        eng.sync()
        res = eng.fetch()
    compare(res, ref, check_counts=False)


def test_counts_exact_default_config(case):
    from gtpower_b200 import B200Power
    d, ev, ref = case
    with B200Power(d, device=0, collect_counts=True) as eng:
        eng.read_power_activities(ev)
        eng.sync()
        assert eng.clock_run_nets() == (1, 1)
        res = eng.fetch(counts=True)
    compare(res, ref, check_counts=True)
    assert res.counts.dropped == ref.dropped
