"""Periodic clock pins walked as runs of whole cycles (the default) against
the FP64 oracle and against the edge-by-edge walk: clocks of several phases
and duties, falling-first clocks, a stopped clock, a clock that is X until
its first edge, data events on clock edges, outputs related to the clock, a
trace ending mid-cycle, windows (on and off cycle boundaries) and tiles of a
few cycles.

Internal and switching energies enter the per-cycle bins as the same 64-bit
fixed-point terms either way, so those columns must agree bit for bit
between the two walks; leakage per cycle is summed per cycle instead of per
edge and agrees within the parity tolerance."""
import numpy as np
import pytest

from tests import toy
from tests.parity import compare

pytestmark = pytest.mark.gpu

TPC = 500
# clock nets walked as runs when the whole trace is one window: a stopped
# clock and a clock that is X before its first edge are walked edge by edge
PERIODIC_ONE_WINDOW = [1, 2, 0, 2]
CLOCKS = [
    # falls at the cycle start, rises mid-cycle (the synthetic designs' clock)
    [dict(pa=0, pb=250, v0=1)],
    # a one-tick pulse; a falling-first clock with a long high phase
    [dict(pa=100, pb=101, v0=0), dict(pa=30, pb=480, v0=1)],
    # a clock stopped for cycles 10..13; a clock that is X until its first edge
    [dict(pa=30, pb=480, v0=0, gap=(10, 14)), dict(pa=200, pb=300, v0=1, initial=False)],
    # edges at both ends of the cycle
    [dict(pa=0, pb=1, v0=0), dict(pa=498, pb=499, v0=1)],
]


def _design(case, n_cycle=40):
    rng = np.random.default_rng(100 + case)
    return toy.clocked_design(rng, n_dff=80, n_comb=40, n_data=30, tpc=TPC, n_cycle=n_cycle,
                              clocks=CLOCKS[case], tail=180 if case % 2 else 0)


def _run(design, windows, clock_runs, periodic=None, **kw):
    """Engine results; `periodic`: the number of clock nets the last window
    must have walked as runs (checked when not None)."""
    from gtpower_b200 import B200Power
    with B200Power(design, collect_counts=True, clock_runs=clock_runs, **kw) as eng:
        for w in windows:
            eng.read_power_activities(w)
        eng.sync()
        n_clk, n_per = eng.clock_run_nets()
        assert n_clk > 0
        if not clock_runs:
            assert n_per == 0
        elif periodic is not None:
            assert n_per == periodic, (n_per, periodic)
        return eng.fetch(counts=True)


def _oracle(design, events):
    from oracle import oracle as orc
    return orc.run(design, events)


def _same_dynamic(a, b):
    # columns 1..4: internal, glitch internal, switching, glitch switching
    assert np.array_equal(a.cycle5[1:], b.cycle5[1:])


@pytest.mark.parametrize("case", range(len(CLOCKS)))
@pytest.mark.parametrize("cycles_per_tile", [0, 1, 3, 7])
def test_clock_runs_match_oracle(case, cycles_per_tile):
    d, ev = _design(case)
    ref = _oracle(d, ev)
    a = _run(d, [ev], True, periodic=PERIODIC_ONE_WINDOW[case], cycles_per_tile=cycles_per_tile)
    b = _run(d, [ev], False, cycles_per_tile=cycles_per_tile)
    compare(a, ref)
    compare(b, ref)
    _same_dynamic(a, b)


@pytest.mark.parametrize("case", range(len(CLOCKS)))
def test_clock_runs_windows_on_cycle_boundaries(case):
    from gtpower_b200 import windows
    d, ev = _design(case)
    wins = windows.split(ev, TPC, [0, 3, 11, 12, 20, 31, 41])
    ref = _oracle(d, ev)
    # the last window (cycles 31..40) holds every clock's context
    a = _run(d, wins, True, periodic=len(CLOCKS[case]), cycles_per_tile=4)
    b = _run(d, wins, False, cycles_per_tile=4)
    compare(a, ref)
    compare(b, ref)
    _same_dynamic(a, b)


@pytest.mark.parametrize("case", range(len(CLOCKS)))
def test_clock_runs_windows_inside_cycles(case):
    """Windows that start between a clock's two edges (the window's first
    edge is the cycle's second one) or right on an edge."""
    from gtpower_b200 import windows
    d, ev = _design(case)
    cuts = [0, 3 * TPC + 250, 7 * TPC + 101, 12 * TPC + 30, 12 * TPC + 490, 25 * TPC + 1, np.iinfo(np.int64).max]
    wins = [windows.make_window(ev, TPC, cuts[k], cuts[k + 1]) for k in range(len(cuts) - 1)]
    ref = _oracle(d, ev)
    b = _run(d, wins, False, cycles_per_tile=5)
    compare(b, ref)
    a = _run(d, wins, True, periodic=len(CLOCKS[case]), cycles_per_tile=5)
    compare(a, ref)
    _same_dynamic(a, b)


def test_clock_runs_on_synthetic_flat_design():
    """The synthetic flat designs' flip-flops (one clock net, 3-pin cells); the
    trace ends at time_max = 90 cycles without the clock edge there."""
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=3000, n_cycle=90, seed=21))
    ev = synth.Trace(d, info, synth.TraceSpec(glitch_p=0.1), seed=22).full()
    ref = _oracle(d, ev)
    a = _run(d, [ev], True, periodic=1)
    b = _run(d, [ev], False)
    compare(a, ref)
    compare(b, ref)
    _same_dynamic(a, b)


@pytest.mark.parametrize("threads,gates", [(128, 0), (64, 256), (256, 1024)])
def test_clock_runs_block_shapes(threads, gates):
    """Blocks of 64 or 128 threads (the run scan with 2 or 4 warps) and
    several cells per thread (the run state and shared sums reset per
    cell)."""
    d, ev = _design(1)
    ref = _oracle(d, ev)
    a = _run(d, [ev], True, periodic=PERIODIC_ONE_WINDOW[1], cycles_per_tile=6, threads_per_block=threads,
             gates_per_block=gates)
    b = _run(d, [ev], False, cycles_per_tile=6, threads_per_block=threads, gates_per_block=gates)
    compare(a, ref)
    compare(b, ref)
    _same_dynamic(a, b)
