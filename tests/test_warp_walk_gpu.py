"""The warp walk (one warp per cell and tile, 32 events at a time in time
order; cells of up to 4 pins without drift) against the per-thread walk and
the FP64 oracle.

Both walks add the same integer fixed-point terms to the per-cycle bins, so
per-cycle results must be bit-identical and counts equal; per-cell FP64 sums
differ only in summation order. Cases: X/Z values, nets whose first event
comes after tick 0, same-time events on several pins, flip-flops on
periodic clocks (runs) and on stopped clocks, windows on and off cycle
boundaries, windows after gaps, cycle groups, tiles of a few cycles."""
import numpy as np
import pytest

from tests import toy
from tests.parity import close, compare

pytestmark = pytest.mark.gpu


def _run(d, windows, groups=None, **kw):
    from gtpower_b200 import B200Power
    with B200Power(d, device=0, collect_counts=True, **kw) as eng:
        if groups is not None:
            eng.set_cycle_groups(groups, int(groups.max()) + 1)
        for w in windows:
            eng.read_power_activities(w)
        eng.sync()
        res = eng.fetch(counts=True)
        cg = eng.fetch_cycle_groups() if groups is not None else None
        return res, cg


def _same(a, b):
    assert np.array_equal(a.cycle5, b.cycle5)
    for f in ("cell_events", "cell_glitches", "cell_half_toggles", "cell_related", "cycle_events",
              "cycle_glitches"):
        assert np.array_equal(getattr(a.counts, f), getattr(b.counts, f)), f
    close("cell5", a.cell5, b.cell5, rtol=1e-9)


@pytest.mark.parametrize("seed,tpc,ct", [(1, 700, 0), (2, 300, 7), (3, 1000, 3), (4, 450, 64)])
def test_random_toy_designs(seed, tpc, ct):
    from oracle import oracle as orc
    rng = np.random.default_rng(seed)
    d, ev = toy.random_design(rng, n_cell=600, n_net=160, time_max=40_000, tpc=tpc, max_events=120)
    ww, _ = _run(d, [ev], cycles_per_tile=ct, warp_walk=True)
    pt, _ = _run(d, [ev], cycles_per_tile=ct)
    _same(ww, pt)
    compare(ww, orc.run(d, ev))


def test_dense_pins_many_chunks():
    """Cells whose pins carry hundreds of events per tile (many 32-event
    chunks, time groups split across chunks by same-time events)."""
    from oracle import oracle as orc
    rng = np.random.default_rng(11)
    d, ev = toy.random_design(rng, n_cell=80, n_net=12, time_max=60_000, tpc=5000, max_events=2000,
                              wide=False)
    ww, _ = _run(d, [ev], warp_walk=True)
    pt, _ = _run(d, [ev])
    _same(ww, pt)
    compare(ww, orc.run(d, ev))


def test_clocked_design_runs_and_windows():
    from gtpower_b200 import windows
    from oracle import oracle as orc
    rng = np.random.default_rng(5)
    d, ev = toy.clocked_design(rng, n_dff=120, n_comb=60, n_data=30, tpc=500, n_cycle=80,
                               clocks=[dict(pa=30, pb=480, v0=0, gap=(10, 14)), dict(pa=100, pb=101, v0=0),
                                       dict(pa=250, pb=499, v0=1)])
    tpc = d.ticks_per_cycle
    cuts = [0, 17 * tpc, 40 * tpc + 123, 61 * tpc, np.iinfo(np.int64).max]
    wins = [windows.make_window(ev, tpc, cuts[k], cuts[k + 1]) for k in range(len(cuts) - 1)]
    for w_list in ([ev], wins):
        ww, _ = _run(d, w_list, cycles_per_tile=9, warp_walk=True)
        pt, _ = _run(d, w_list, cycles_per_tile=9)
        _same(ww, pt)
        compare(ww, orc.run(d, ev))


def test_flat_synthetic_with_groups_and_gaps():
    from gtpower_b200 import synth, windows
    d, info = synth.flat_design(synth.FlatSpec(n_cell=4000, n_cycle=160, seed=91))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, zipf_alpha=1.2, rate_mean=0.1, burst_sigma=1.5,
                                             glitch_p=0.1), seed=92).full()
    tpc = d.ticks_per_cycle
    groups = (np.arange(d.n_cell) * 9 // d.n_cell).astype(np.int32)
    spans = [(0, 30), (33, 34), (40, 101), (110, None)]
    wins = [windows.make_window(ev, tpc, c0 * tpc, c1 * tpc if c1 else np.iinfo(np.int64).max)
            for c0, c1 in spans]
    ww, cw = _run(d, wins, groups=groups, warp_walk=True)
    pt, cp = _run(d, wins, groups=groups)
    _same(ww, pt)
    assert np.array_equal(cw, cp)


def test_time_order_error_reported():
    from gtpower_b200 import B200Power, _abi
    from gtpower_b200.design import Events
    rng = np.random.default_rng(2)
    d, ev = toy.random_design(rng, n_cell=60, n_net=20, time_max=5_000, tpc=500, wide=False)
    t = ev.time.copy()
    counts = np.diff(ev.net_off)
    n = next(int(x) for x in np.unique(d.pin_net[d.pin_net >= 0]) if counts[x] >= 4)
    a = int(ev.net_off[n])
    t[a + 2] = t[a + 1]
    bad = Events.from_values(ev.net_off, t, ev.values())
    with B200Power(d, device=0, warp_walk=True) as eng:
        eng.read_power_activities(bad)
        with pytest.raises(_abi.GtpError) as exc:
            eng.sync()
        assert "strictly increasing" in str(exc.value)
        eng.reset()
        eng.read_power_activities(ev)
        eng.sync()
