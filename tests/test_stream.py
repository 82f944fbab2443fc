"""Streaming windows: every listed event of every window is the event at
the same index (net_base + j) of the whole trace, windows tile the trace,
and each window carries the head context the walk reads."""
import numpy as np
import pytest


@pytest.mark.parametrize("window", [1, 7, 13, 200])
def test_stream_windows_are_slices_of_the_trace(window):
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=600, n_cycle=70, seed=4))
    spec = synth.TraceSpec(mode=1, glitch_p=0.1)
    full = synth.Trace(d, info, spec, seed=9).full()
    fv = full.values()
    st = synth.Stream(synth.Trace(d, info, spec, seed=9), window)
    tpc = d.ticks_per_cycle
    t_prev = 0
    covered = np.zeros(full.n_event, bool)
    while True:
        w = st.next(100_000)
        if w is None:
            break
        assert w.t_lo == t_prev
        wv = w.values()
        for n in range(d.n_net):
            a, b = int(w.net_off[n]), int(w.net_off[n + 1])
            fa = int(full.net_off[n] + w.net_base[n])
            assert np.array_equal(w.time[a:b], full.time[fa:fa + b - a])
            assert np.array_equal(wv[a:b], fv[fa:fa + b - a])
            inside = (w.time[a:b] >= w.t_lo) & (w.time[a:b] < w.t_hi)
            covered[fa:fa + b - a] |= inside
            # head context: the event before t_lo is listed when one exists
            before = full.time[full.net_off[n]:full.net_off[n + 1]] < w.t_lo
            if before.any():
                assert (w.time[a:b] < w.t_lo).any()
        t_prev = w.t_hi if w.t_hi != np.iinfo(np.int64).max else t_prev
        assert w.t_lo % tpc == 0
    assert covered.all()
