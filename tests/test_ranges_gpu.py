"""Spot evaluation of selected cycles against the FP64 oracle of the whole
trace: cycle ranges of one window in one pass
(gtp_push_events_device_ranges), and windows pushed with gaps between them.

In both, a range or window is evaluated on its own: its state comes from the
events listed before it, its leakage starts at its first tick and ends at
its last. Per-cycle power and counts inside the evaluated cycles must equal
the oracle's over the whole trace (leakage included); outside them they are
zero."""
import numpy as np
import pytest

from tests import toy
from tests.parity import close

pytestmark = pytest.mark.gpu


def _has_drift(d) -> bool:
    """Tick and seconds cycle boundaries disagree somewhere (the engine's rule)."""
    P = float(np.float32(d.clk_period))
    tpc = d.ticks_per_cycle
    for c in range(1, d.n_period + 2):
        b = c * P
        t0 = c * tpc
        if not (b <= t0 * d.timescale) or (b <= (t0 - 1) * d.timescale):
            return True
    return False


def _check(res, ref, cycles):
    mask = np.zeros(ref.cycle5.shape[1], dtype=bool)
    for c0, c1 in cycles:
        mask[c0:c1] = True
    close("cycle5 in ranges", res.cycle5[:, mask].T, ref.cycle5[:, mask].T)
    assert np.all(res.cycle5[:, ~mask] == 0)
    assert np.array_equal(res.counts.cycle_events[mask], ref.cycle_events[mask])
    assert np.array_equal(res.counts.cycle_glitches[mask], ref.cycle_glitches[mask])
    assert np.all(res.counts.cycle_events[~mask] == 0)


@pytest.fixture(scope="module")
def flat():
    from gtpower_b200 import synth
    from oracle import oracle as orc
    d, info = synth.flat_design(synth.FlatSpec(n_cell=2500, n_cycle=120, seed=71))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=0.1), seed=72).full()
    assert not _has_drift(d)
    return d, ev, orc.run(d, ev)


def _device(ev):
    import torch
    dev = torch.device("cuda", 0)
    return [torch.from_numpy(a).to(dev) for a in (ev.net_off, ev.time, ev.packed.view(np.int32))]


@pytest.mark.parametrize("cycles_per_tile", [0, 4])
def test_cycle_ranges_one_pass(flat, cycles_per_tile):
    from gtpower_b200 import B200Power
    d, ev, ref = flat
    ranges = [(0, 2), (3, 9), (40, 41), (77, 100), (119, 120)]
    t = _device(ev)
    with B200Power(d, device=0, collect_counts=True, cycles_per_tile=cycles_per_tile) as eng:
        eng.push_device_ranges(ev.n_event, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), ranges)
        eng.sync()
        res = eng.fetch(counts=True)
    _check(res, ref, ranges)


def test_windows_with_gaps(flat):
    from gtpower_b200 import B200Power, windows
    d, ev, ref = flat
    tpc = d.ticks_per_cycle
    spans = [(5, 30), (50, 51), (60, 95), (101, None)]
    wins = [windows.make_window(ev, tpc, c0 * tpc, c1 * tpc if c1 else np.iinfo(np.int64).max)
            for c0, c1 in spans]
    with B200Power(d, device=0, collect_counts=True) as eng:
        for w in wins:
            eng.read_power_activities(w)
        eng.sync()
        res = eng.fetch(counts=True)
    # the last window runs to the trace's end, including the sliver of a
    # cycle past 120 x 2 ns that the float period leaves before time_max
    _check(res, ref, [(c0, c1 or d.n_period) for c0, c1 in spans])


def test_ranges_on_clocked_design():
    """Flip-flops on periodic and stopped clocks (walked edge by edge in a
    range push), ranges starting between a clock's two edges' cycles."""
    from gtpower_b200 import B200Power
    from oracle import oracle as orc
    rng = np.random.default_rng(5)
    d, ev = toy.clocked_design(rng, n_dff=60, n_comb=30, n_data=20, tpc=500, n_cycle=40,
                               clocks=[dict(pa=30, pb=480, v0=0, gap=(10, 14)), dict(pa=100, pb=101, v0=0)])
    if _has_drift(d):
        pytest.skip("design has tick/seconds drift")
    ref = orc.run(d, ev)
    ranges = [(1, 4), (9, 15), (33, 40)]
    t = _device(ev)
    with B200Power(d, device=0, collect_counts=True) as eng:
        eng.push_device_ranges(ev.n_event, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), ranges)
        eng.sync()
        res = eng.fetch(counts=True)
    _check(res, ref, ranges)


def test_bad_ranges_rejected(flat):
    from gtpower_b200 import B200Power, _abi
    d, ev, _ = flat
    t = _device(ev)
    with B200Power(d, device=0) as eng:
        for bad in ([(5, 5)], [(9, 12), (10, 20)], [(20, 10)]):
            with pytest.raises(_abi.GtpError):
                eng.push_device_ranges(ev.n_event, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), bad)


def test_ranges_with_drift():
    """A period of 300.5 ticks: cycles of 301 ticks drift half a tick a cycle
    away from the seconds boundaries. Dynamic power and counts of the range
    cycles are exact; leakage too except in the cycles that straddle a
    range's edge in seconds, where the range covers its part only."""
    from gtpower_b200 import B200Power
    from oracle import oracle as orc
    rng = np.random.default_rng(1)
    d, ev = toy.random_design(rng, n_cell=120, n_net=40, time_max=15_000, tpc=300, wide=False)
    d.clk_period = 300.5e-12
    assert _has_drift(d)
    ref = orc.run(d, ev)
    ranges = [(3, 12), (20, 31), (40, d.n_period)]
    t = _device(ev)
    with B200Power(d, device=0, collect_counts=True) as eng:
        eng.push_device_ranges(ev.n_event, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), ranges)
        eng.sync()
        res = eng.fetch(counts=True)
    mask = np.zeros(d.n_period, bool)
    inner = np.zeros(d.n_period, bool)
    for c0, c1 in ranges:
        mask[c0:c1] = True
        inner[c0 + 1:c1 - 1] = True
    close("dynamic in ranges", res.cycle5[1:, mask].T, ref.cycle5[1:, mask].T)
    close("leakage inside ranges", res.cycle5[0, inner], ref.cycle5[0, inner])
    # a range starting at cycle c0 misses the 0.5 * c0 ticks of seconds
    # cycle c0 that lie before its first tick (at the cells' states then,
    # whose leakage may lie above the cycle's mean)
    for c0, _ in ranges:
        miss = 0.5 * c0 / 300.5
        assert abs(res.cycle5[0, c0] - ref.cycle5[0, c0]) <= 2 * miss * abs(ref.cycle5[0, c0]) + 1e-30
    assert np.array_equal(res.counts.cycle_events[mask], ref.cycle_events[mask])
    assert np.all(res.cycle5[1:, ~mask] == 0)
