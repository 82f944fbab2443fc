"""Host-pushed windows walk on two alternating streams, each with its own
walk scratch, so that a window's walk may overlap the tail of the one
before. These tests mix them with the context's own stream: device-pushed
windows, resets and fetches without a sync in between must see the same
results as the plain orders."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _trace(d, info, seed, glitch_p):
    from gtpower_b200 import synth
    return synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=glitch_p), seed=seed).full()


def _case(seed, n_cell=6000, n_cycle=240, glitch_p=0.1):
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=n_cell, n_cycle=n_cycle, seed=seed))
    return d, _trace(d, info, seed + 1, glitch_p)


def _windows(d, ev, n):
    from gtpower_b200 import windows as W
    tpc = d.ticks_per_cycle
    cuts = np.linspace(0, d.n_period, n + 1).astype(np.int64) * tpc
    cuts[-1] = np.iinfo(np.int64).max
    return [W.make_window(ev, tpc, int(cuts[k]), int(cuts[k + 1])) for k in range(n)]


def _device(w):
    import torch
    arrs = [torch.from_numpy(np.ascontiguousarray(a)).cuda()
            for a in (w.net_off, w.time, w.packed.view(np.int32), w.net_base)]
    return w.n_event, arrs, w.t_lo, w.t_hi


def _push(eng, w, dev):
    if dev is None:
        eng.read_power_activities(w)
    else:
        n, a, lo, hi = dev
        eng.push_device(n, a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr(), a[3].data_ptr(), lo, hi)


def _same(a, b):
    assert np.array_equal(a.cycle5, b.cycle5)
    assert np.array_equal(a.counts.cell_events, b.counts.cell_events)
    assert np.array_equal(a.counts.cycle_events, b.counts.cycle_events)
    np.testing.assert_allclose(a.cell5, b.cell5, rtol=1e-12, atol=0)


def test_host_and_device_windows_interleaved():
    from gtpower_b200 import B200Power
    d, ev = _case(71)
    wins = _windows(d, ev, 7)
    devs = [_device(w) for w in wins]
    orders = {
        "host": [None] * len(wins),
        "device": devs,
        "alternating": [dv if k % 2 else None for k, dv in enumerate(devs)],
        "device first": [dv if k < 2 else None for k, dv in enumerate(devs)],
    }
    out = {}
    for name, how in orders.items():
        with B200Power(d, device=0, collect_counts=True) as eng:
            for w, dv in zip(wins, how):
                _push(eng, w, dv)
            out[name] = eng.fetch(counts=True)   # no sync before the fetch
    for name in orders:
        _same(out[name], out["host"])


def test_reset_between_traces_without_sync():
    """Two traces on one context, reset in between with walks in flight: the
    second trace's results are a fresh context's."""
    from gtpower_b200 import B200Power, synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=6000, n_cycle=240, seed=81))
    ev1, ev2 = _trace(d, info, 82, 0.1), _trace(d, info, 99, 0.2)
    w1, w2 = _windows(d, ev1, 6), _windows(d, ev2, 5)
    with B200Power(d, device=0, collect_counts=True) as fresh:
        for w in w2:
            fresh.read_power_activities(w)
        ref = fresh.fetch(counts=True)
    with B200Power(d, device=0, collect_counts=True) as eng:
        for rep in range(2):
            for w in w1:
                eng.read_power_activities(w)
            eng.reset()
            for w in w2:
                eng.read_power_activities(w)
            got = eng.fetch(counts=True)
            _same(got, ref)
            eng.reset()


def test_windows_match_the_oracle_with_overlap():
    """Many small windows (each walk short, so consecutive walks overlap the
    most) against the FP64 oracle."""
    from gtpower_b200 import B200Power
    from oracle import oracle as orc
    from tests.parity import compare
    d, ev = _case(91, n_cell=4000, n_cycle=300, glitch_p=0.15)
    with B200Power(d, device=0, collect_counts=True) as eng:
        for w in _windows(d, ev, 15):
            eng.read_power_activities(w)
        got = eng.fetch(counts=True)
    compare(got, orc.run(d, ev))
