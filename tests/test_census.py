"""Divergence census of the reference's two implementations of the path.

The reference ships a CPU path (power/TimeBasedPower.cc), which this package
follows, and a CUDA path (power/cuda/CudaPower.cu:317-584) that decides some
events differently. oracle.divergence_census walks the CPU path and counts
the events on which the CUDA rules would decide otherwise. Each case below
plants one such event in a one-cell design and checks the exact counts;
the last tests pin the counts on the GCD example tape.
"""
import os

import numpy as np

import toy
from gtpower_b200.design import GROUP_SEQUENTIAL

HERE = os.path.dirname(os.path.abspath(__file__))

ZERO = dict(same_tick_state=0, same_tick_energy=0, first_event_state=0, glitch_class_diff=0,
            glitch_width_diff=0, related_diff=0, no_group_match=0, beyond_cuda_cycles=0, z_events=0)


def census(d, ev):
    from oracle import oracle as orc
    return orc.divergence_census(d, ev, threads=1)


def expect(c, pin_events, toggles, **kw):
    want = dict(ZERO, pin_events=pin_events, toggles=toggles, **kw)
    assert c == want


def test_same_tick_lookup_with_new_values():
    # NAND2W: A's input tables depend on B (B=1: 7 fJ, B=0: 5 fJ). B sits on
    # net 0, so its event index is lower and the CUDA kernel walks it first:
    # A's lookup then sees B=1 where the CPU path uses the state before the tick.
    d = toy.build([toy.nand_cell("NAND2W", when_tables=True)], [(0, [1, 0, 2])], 3, time_max=2000)
    ev = toy.events(3, {0: [(0, 0), (100, 1)], 1: [(0, 0), (100, 1)]})
    expect(census(d, ev), 2, 2, same_tick_state=1, same_tick_energy=1)


def test_same_tick_lookup_state_only():
    # the other order: B's lookup sees A's new value, but B's tables do not
    # depend on A, so the energy is the same
    d = toy.build([toy.nand_cell("NAND2W", when_tables=True)], [(0, [0, 1, 2])], 3, time_max=2000)
    ev = toy.events(3, {0: [(0, 0), (100, 1)], 1: [(0, 0), (100, 1)]})
    expect(census(d, ev), 2, 2, same_tick_state=1)


def test_first_event_after_zero():
    # A's net starts at t=50: the CPU path walks X -> 1 there, the CUDA
    # kernel starts from state 1
    d = toy.build([toy.inv_cell()], [(0, [0, 1])], 2, time_max=2000)
    ev = toy.events(2, {0: [(50, 1), (200, 0)]})
    expect(census(d, ev), 2, 2, first_event_state=1)


def test_glitch_class_non_toggling_neighbour():
    # period 1 holds a rise, a repeated 1 and a fall. The CPU path flags the
    # first two of the three events; the CUDA counters skip the repeated
    # value, count the fall as the period's second toggle and keep its
    # width to the repeated event.
    d = toy.build([toy.inv_cell()], [(0, [0, 1])], 2, time_max=3000)
    ev = toy.events(2, {0: [(0, 0), (1100, 1), (1200, 1), (1300, 0)]})
    expect(census(d, ev), 3, 2, glitch_class_diff=1)


def test_glitch_width_initial_event():
    # t=0, 30, 40 in one period: the CPU path never flags the initial event,
    # the CUDA rule takes the 30-tick gap to it as the rise's pulse width
    d = toy.build([toy.inv_cell()], [(0, [0, 1])], 2, time_max=2000)
    ev = toy.events(2, {0: [(0, 0), (30, 1), (40, 0)]})
    expect(census(d, ev), 2, 2, glitch_width_diff=1)


def test_related_near_tie():
    # A and B rise together and Y falls 10 ticks later, the arc delay: both
    # are exact. The CPU path keeps the first (A), the CUDA near-tie rule the
    # later event index (B). B's lookup also sees A's new value.
    d = toy.build([toy.nand_cell()], [(0, [0, 1, 2])], 3, time_max=2000)
    ev = toy.events(3, {0: [(0, 0), (100, 1)], 1: [(0, 0), (100, 1)], 2: [(0, 1), (110, 0)]})
    expect(census(d, ev), 3, 3, same_tick_state=1, related_diff=1)


def test_related_same_cycle_rule_logic_cells_only():
    # a flip-flop whose Q toggles in cycle 1 while its inputs last moved in
    # cycle 0: the CPU path finds no related pin, the CUDA kernel applies the
    # same-cycle rule to combinational cells only and relates Q to D
    d = toy.build([toy.dff_cell()], [(0, [0, 1, 2])], 3, time_max=3000, clock_pins=[1],
                  groups=[GROUP_SEQUENTIAL])
    ev = toy.events(3, {0: [(0, 1), (500, 0)], 1: [(0, 0), (600, 1)], 2: [(0, 0), (1005, 1)]})
    expect(census(d, ev), 3, 3, related_diff=1)


def test_output_without_matching_group():
    # Y's table holds only when A=1; Y rises just after A fell: the CPU path
    # gives no energy, the CUDA kernel the default average
    cell = toy.inv_cell()
    cell["internal_powers"][1]["when"] = [[1, 1]]
    d = toy.build([cell], [(0, [0, 1])], 2, time_max=2000)
    ev = toy.events(2, {0: [(0, 1), (100, 0)], 1: [(0, 0), (110, 1)]})
    expect(census(d, ev), 2, 2, no_group_match=1)


def test_event_past_last_cuda_cycle():
    # time_max 10000 ticks, 1000 ticks a cycle: an event at 10000 is in cycle
    # 10. The CUDA kernel's last thread ends one tick past cycle 10's start,
    # so it walks the event, and adds its per-cycle terms past its 10 entries
    d = toy.build([toy.inv_cell()], [(0, [0, 1])], 2, time_max=10_000)
    ev = toy.events(2, {0: [(0, 0), (10_000, 1)]})
    expect(census(d, ev), 1, 1, beyond_cuda_cycles=1)


def test_z_toggle():
    d = toy.build([toy.inv_cell()], [(0, [0, 1])], 2, time_max=2000)
    ev = toy.events(2, {0: [(0, 0), (100, 3)]})
    expect(census(d, ev), 1, 1, z_events=1)


def test_census_walk_leaves_results_unchanged():
    # the census rides on the FP64 walk; the oracle's outputs with and
    # without it are the same walk, so the event totals agree
    from oracle import oracle as orc
    rng = np.random.default_rng(7)
    d, ev = toy.random_design(rng, 40, 60, 8000, 700)
    c = orc.divergence_census(d, ev, threads=3)
    r = orc.run(d, ev)
    assert c["pin_events"] == int(r.cell_events.sum())
    assert c["toggles"] <= c["pin_events"]
    assert c["same_tick_energy"] <= c["same_tick_state"]
    assert orc.divergence_census(d, ev, threads=1) == c


def test_gcd_exposure():
    # the reference's GCD example: 5793 toggles, of which 10 get another
    # glitch pulse width and 45 lie at the trace's end tick (t = 125000,
    # cycle 25: the CPU path's 26th per-cycle entry, one past the CUDA
    # kernel's 25); 1215 input lookups at shared ticks see other states,
    # none with another energy
    from gtpower_b200 import tape
    from oracle import oracle as orc
    d, ev, _ = tape.load(os.path.join(HERE, "golden", "gcd_tape.npz"))
    c = orc.divergence_census(d, ev, threads=2)
    expect(c, 5793, 5793, same_tick_state=1215, glitch_width_diff=10, beyond_cuda_cycles=45)
