"""Window splits of a trace: the e2e leg's (bench.e2e_cuts: windows growing
by a ramp, covering every cycle once, in order, and together listing every
event of the trace) and the reference's event-count intervals
(windows.interval_edges, split_by_events)."""
import numpy as np
import pytest


@pytest.mark.parametrize("cycles", [1, 7, 100, 10_000])
@pytest.mark.parametrize("windows", [1, 2, 8, 12, 30])
@pytest.mark.parametrize("ramp", [1.0, 1.25, 1.5, 2.0])
def test_cuts_cover_the_trace(cycles, windows, ramp):
    import bench
    cuts = bench.e2e_cuts(cycles, windows, ramp)
    assert cuts[0] == 0 and cuts[-1] == cycles
    assert np.all(np.diff(cuts) > 0)
    assert len(cuts) - 1 <= windows


def test_default_split_grows():
    import bench
    cuts = bench.e2e_cuts(10_000, 12, 1.25)
    sizes = np.diff(cuts)
    assert len(sizes) == 12
    assert np.all(np.diff(sizes) >= 0)
    # the first copy is about 1.5% of the trace, the last window about 25%
    assert 100 <= sizes[0] <= 300 and 2000 <= sizes[-1] <= 3000


def test_windows_list_every_event_once():
    import bench
    from gtpower_b200 import synth, windows as W
    d, info = synth.flat_design(synth.FlatSpec(n_cell=300, n_cycle=97, seed=5))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=0.2), seed=6).full()
    tpc = d.ticks_per_cycle
    cuts = bench.e2e_cuts(97, 9, 1.25)
    seen = 0
    for k in range(len(cuts) - 1):
        lo = int(cuts[k]) * tpc
        hi = int(cuts[k + 1]) * tpc if k + 2 < len(cuts) else np.iinfo(np.int64).max
        w = W.make_window(ev, tpc, lo, hi)
        seen += int(np.count_nonzero((w.time >= lo) & (w.time < hi)))
    assert seen == ev.n_event


def _reference_rule(times, tpc, max_events):
    # the running count of listed events in time order; the interval ends at
    # the time of the event that takes it past max_events, and counting
    # starts again after that event; bounds rounded up to cycles
    edges, count = [0], 0
    for t in sorted(times):
        count += 1
        if count > max_events:
            c = -(-int(t) // tpc)
            if c > edges[-1]:
                edges.append(c)
            count = 0
    last = int(max(times)) // tpc + 1
    if last > edges[-1]:
        edges.append(last)
    return edges


@pytest.mark.parametrize("max_events", [1, 7, 50, 400, 10**6])
def test_interval_edges_follow_the_reference_rule(max_events):
    from gtpower_b200 import synth, windows as W
    d, info = synth.flat_design(synth.FlatSpec(n_cell=200, n_cycle=60, seed=9))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=0.1), seed=10).full()
    tpc = d.ticks_per_cycle
    edges = W.interval_edges(ev, tpc, max_events)
    assert edges == _reference_rule(ev.time.tolist(), tpc, max_events)
    assert edges[0] == 0 and all(b > a for a, b in zip(edges, edges[1:]))
    wins = W.split_by_events(ev, tpc, max_events)
    assert len(wins) == len(edges) - 1
    seen = sum(int(np.count_nonzero((w.time >= w.t_lo) & (w.time < w.t_hi))) for w in wins)
    assert seen == ev.n_event
