"""Density-aware split of the walk against the FP64 oracle.

Per window the engine measures each cell's event count (its pins' listed
events, periodic clock pins excluded) and, as the reference's
cycles-per-thread rule does (power/cuda/Gate.cuh:354-376), gives a cell
whose events per cycle tile exceed split_events several threads, each over
an equal share of the tile's cycles. The tests force low thresholds on
skewed traces (Zipf(1.2) net rates, lognormal(1.5) per-cycle bursts, glitch
rate 0.1) so that many cells are split, and compare counts bit for bit and
powers within the parity tolerance; the split must not change a result."""
import numpy as np
import pytest

from tests import toy
from tests.parity import compare

pytestmark = pytest.mark.gpu


def _oracle(d, ev):
    from oracle import oracle as orc
    return orc.run(d, ev)


def _run(d, windows, split_events, **kw):
    from gtpower_b200 import B200Power
    with B200Power(d, device=0, collect_counts=True, split_events=split_events, **kw) as eng:
        for w in windows:
            eng.read_power_activities(w)
        eng.sync()
        items = eng.walk_items()
        return eng.fetch(counts=True), items


@pytest.fixture(scope="module")
def skew():
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=3000, n_cycle=300, seed=41))
    spec = synth.TraceSpec(mode=1, zipf_alpha=1.2, rate_mean=0.1, burst_sigma=1.5, glitch_p=0.1)
    ev = synth.Trace(d, info, spec, seed=42).full()
    return d, ev, _oracle(d, ev)


@pytest.mark.parametrize("split_events,cycles_per_tile", [(8, 0), (32, 0), (16, 64), (4, 7)])
def test_split_skewed_trace(skew, split_events, cycles_per_tile):
    d, ev, ref = skew
    res, items = _run(d, [ev], split_events, cycles_per_tile=cycles_per_tile)
    assert items > d.n_cell            # some cells were walked by several threads
    compare(res, ref)


def test_split_off_and_default_agree(skew):
    d, ev, ref = skew
    off, items_off = _run(d, [ev], -1)
    assert items_off == 0
    dflt, items = _run(d, [ev], 0)
    assert items == d.n_cell           # nothing this light passes 2048 events per tile
    compare(off, ref)
    compare(dflt, ref)
    # the integer per-cycle bins of the dynamic quantities do not depend on
    # how the cycles were shared out
    low, _ = _run(d, [ev], 8)
    assert np.array_equal(low.cycle5[1:], off.cycle5[1:])


def test_split_windows_and_clock_runs(skew):
    """Windows on and off cycle boundaries, the clock net on runs, cells
    split across both."""
    from gtpower_b200 import windows
    d, ev, ref = skew
    tpc = d.ticks_per_cycle
    cuts = [0, 37 * tpc, 90 * tpc + 333, 211 * tpc, np.iinfo(np.int64).max]
    wins = [windows.make_window(ev, tpc, cuts[k], cuts[k + 1]) for k in range(len(cuts) - 1)]
    res, items = _run(d, wins, 8, cycles_per_tile=32)
    assert items > d.n_cell
    compare(res, ref)


@pytest.mark.parametrize("seed", [1, 2])
def test_split_random_toy_designs(seed):
    """X/Z values, wide cells (8- and 32-pin buckets), pins without nets,
    same-time events, with every cell split."""
    rng = np.random.default_rng(seed)
    d, ev = toy.random_design(rng, n_cell=300, n_net=120, time_max=20_000, tpc=700)
    res, items = _run(d, [ev], 1, cycles_per_tile=9)
    assert items > d.n_cell
    compare(res, _oracle(d, ev))
