"""Known-answer tests of the CPU oracle on hand-built cells.

Every expected value below is derived by hand from the reference's rules
(power/TimeBasedPower.cc, power/PowerUtils.cc, liberty/TableModel.cc), not
by calling the oracle's code, so these tests pin the restatement.

Toy INV (tests/toy.py): leakage 1e-9 W when A, 2e-9 W when !A; input
energy on A: rise = 1-D table over slew {0, 1 ns} -> {1, 3} fJ, fall =
1 fJ; output energy related to A: 2-D (slew, cap) tables; arcs A->Y
negative unate, 10 ps. Slews 0.2 ns rise / 0.3 ns fall, output load 5 fF,
1.8 V. Time base: 1 ps ticks, 1 ns clock (1000 ticks per cycle),
time_max 10000. Liberty values, slews and caps reach the walk as float32,
so expected values round those inputs to float32 and compute in FP64.
"""
import numpy as np
import pytest

from tests import toy

TMAX = 10_000
TS = 1e-12
PF = float(np.float32(1e-9))          # Power::clk_period_ is a float
NORM = TMAX * TS                      # timeMax * timeScale


def f(x):
    return float(np.float32(x))


def approx(x, rel):
    return pytest.approx(x, rel=rel, abs=0)


SR, SF, CAP = f(2e-10), f(3e-10), f(5e-15)
VOLT = f(1.8)


def lerp(x, x0, x1, y0, y1):
    d = (x - f(x0)) / (f(x1) - f(x0))
    return (1 - d) * f(y0) + d * f(y1)


def bilerp(x, y, ax, ay, v):
    """Bilinear interpolation on a 2x2 table v[[x0y0, x0y1], [x1y0, x1y1]]."""
    dx = (x - f(ax[0])) / (f(ax[1]) - f(ax[0]))
    dy = (y - f(ay[0])) / (f(ay[1]) - f(ay[0]))
    return ((1 - dx) * (1 - dy) * f(v[0]) + dx * (1 - dy) * f(v[2]) + dx * dy * f(v[3])
            + (1 - dx) * dy * f(v[1]))


E_IN_RISE = lerp(SR, 0.0, 1e-9, 1e-15, 3e-15)        # A rise at the rise slew
E_IN_FALL = f(1e-15)
OUT_RISE = [1e-14, 2e-14, 3e-14, 5e-14]              # [slew0cap0, slew0cap1, slew1cap0, slew1cap1]
OUT_FALL = [2e-14, 2e-14, 4e-14, 6e-14]


def out_energy(table, slew):
    return bilerp(slew, CAP, [0.0, 1e-9], [0.0, 1e-14], table)


def run(design, ev):
    from oracle import oracle
    return oracle.run(design, ev)


def inv_design(**kw):
    return toy.build([toy.inv_cell()], [(0, [0, 1])], 2, period=1e-9, time_max=TMAX, **kw)


def test_time_base():
    d = inv_design()
    assert d.ticks_per_cycle == 1000
    # ceil(1e-8 / float(1e-9)) = ceil(10.0000003) = 11 entries (power/Power.cc:248)
    assert d.n_period == 11


def test_constant_state_leakage_and_cycle_split():
    d = inv_design()
    ev = toy.events(2, {0: [(0, 1)], 1: [(0, 0)]})
    r = run(d, ev)
    # state A=1 -> 1e-9 W for the whole trace
    assert r.cell5[0, 4] == approx(f(1e-9), rel=1e-12)
    assert np.all(r.cell5[0, :4] == 0)
    # cycles 0..9 are whole clock periods; cycle 10 holds the sliver
    # between 10*P and time_max*ts
    np.testing.assert_allclose(r.cycle5[0, :10], f(1e-9), rtol=1e-12)
    assert r.cycle5[0, 10] == approx(f(1e-9) * (1e-8 - 10 * PF) / PF, rel=1e-6)
    assert r.cell_events[0] == 0 and r.cycle_events.sum() == 0


def test_input_toggle_energy_and_leakage_segments():
    d = inv_design()
    ev = toy.events(2, {0: [(0, 0), (2500, 1)], 1: [(0, 1)]})
    r = run(d, ev)
    assert r.cell5[0, 0] == approx(E_IN_RISE / NORM, rel=1e-12)
    assert r.cycle5[1, 2] == approx(E_IN_RISE / PF, rel=1e-12)
    # leakage: !A (2e-9) for 2500 ticks, then A (1e-9) for 7500
    assert r.cell5[0, 4] == approx((f(2e-9) * 2500 + f(1e-9) * 7500) / TMAX, rel=1e-12)
    # cycle 2 splits at tick 2500
    exp = (f(2e-9) * (2.5e-9 - 2 * PF) + f(1e-9) * (3 * PF - 2.5e-9)) / PF
    assert r.cycle5[0, 2] == approx(exp, rel=1e-9)
    assert (r.cell_events[0], r.cell_glitches[0], r.cell_half_toggles[0], r.cell_related[0]) == (1, 0, 2, 0)
    assert r.cycle_events[2] == 1


def test_output_event_related_pin_and_switching():
    d = inv_design()
    ev = toy.events(2, {0: [(0, 0), (1000, 1), (5000, 0)], 1: [(0, 1), (1010, 0), (5010, 1)]})
    r = run(d, ev)
    e_in = E_IN_RISE + E_IN_FALL
    # Y fall related to A (A rose 10 ticks earlier, arc delay 10 ps): fall
    # table at A's rise slew; Y rise related to A (A fell): rise table at
    # A's fall slew
    e_out = out_energy(OUT_FALL, SR) + out_energy(OUT_RISE, SF)
    assert r.cell5[0, 0] == approx((e_in + e_out) / NORM, rel=1e-12)
    esw = CAP * VOLT * VOLT
    assert r.cell5[0, 2] == approx(esw / NORM, rel=1e-6)
    assert r.cycle5[3, 5] == approx(esw / PF, rel=1e-6)
    assert r.cell_related[0] == 2        # two output events, related pin index 0 -> +1 each
    assert r.cell_events[0] == 4


def default_fall():
    # average over A's rise and fall slews of the fall table
    return (out_energy(OUT_FALL, SR) + out_energy(OUT_FALL, SF)) / 2


def test_default_output_energy_without_arc():
    d = toy.build([toy.inv_cell()], [(0, [0, 1])], 2, period=1e-9, time_max=TMAX,
                  arcs=lambda i, o, q, fr, to: np.nan)
    ev = toy.events(2, {0: [(0, 0)], 1: [(0, 1), (1010, 0)]})
    r = run(d, ev)
    assert r.cell5[0, 0] == approx(default_fall() / NORM, rel=1e-6)
    assert r.cell_related[0] == 0


def test_related_pin_needs_same_cycle():
    d = inv_design()
    # A rose in cycle 0, Y falls in cycle 1: no related pin -> default energy
    ev = toy.events(2, {0: [(0, 0), (990, 1)], 1: [(0, 1), (1005, 0)]})
    r = run(d, ev)
    assert r.cell5[0, 0] == approx((E_IN_RISE + default_fall()) / NORM, rel=1e-6)
    assert r.cell_related[0] == 0


def test_related_pin_uses_event_strictly_before():
    d = inv_design()
    # A and Y change at the same tick: the related search looks at A's last
    # event strictly before (tick 500, a rise) and its arc delay makes it the
    # related pin; Y falls, so the fall table at A's rise slew applies.
    # A's two events share clock period 0, so both are glitch events (pulse
    # 200 ps); Y's single event is not.
    ev = toy.events(2, {0: [(0, 0), (500, 1), (700, 0)], 1: [(0, 1), (700, 0)]})
    r = run(d, ev)
    assert r.cell5[0, 0] == approx(out_energy(OUT_FALL, SR) / NORM, rel=1e-12)
    assert r.cell5[0, 1] == approx(glitch_ratio(200) * (E_IN_RISE + E_IN_FALL) / NORM, rel=1e-6)
    assert r.cell_related[0] == 1 and r.cell_glitches[0] == 2


def glitch_ratio(w_ticks):
    pulse = f(w_ticks * TS)
    return min(1.0, f((pulse * 2.0) / f(SR + SF)) ** 2)


def test_glitch_classification_odd_count():
    d = inv_design()
    # 3 events in cycle 3: the first two are glitch events (k odd -> k-1)
    ev = toy.events(2, {0: [(0, 0), (3100, 1), (3150, 0), (3400, 1)], 1: [(0, 1)]})
    r = run(d, ev)
    g = glitch_ratio(50)
    assert g == approx(0.04, rel=1e-5)
    gl = g * (E_IN_RISE + E_IN_FALL)
    assert r.cell5[0, 1] == approx(gl / NORM, rel=1e-6)
    assert r.cell5[0, 0] == approx(E_IN_RISE / NORM, rel=1e-12)
    assert r.cell_glitches[0] == 2 and r.cell_events[0] == 3
    assert r.cycle_glitches[3] == 2 and r.cycle_events[3] == 3
    # per-cycle internal includes the glitch part
    assert r.cycle5[1, 3] == approx((gl + E_IN_RISE) / PF, rel=1e-6)
    assert r.cycle5[2, 3] == approx(gl / PF, rel=1e-6)


def test_glitch_classification_even_and_neighbouring_periods():
    d = inv_design()
    # cycle 2: two events (both glitch); cycle 3: two events (both glitch).
    # The last of cycle 2 and the first of cycle 3 are flagged neighbours, so
    # their pulse width is the max of both gaps.
    t = [(0, 0), (2100, 1), (2900, 0), (3050, 1), (3080, 0)]
    ev = toy.events(2, {0: t, 1: [(0, 1)]})
    r = run(d, ev)
    w = [800, max(800, 150), max(150, 30), 30]          # widths of events 1..4
    e = [E_IN_RISE, E_IN_FALL, E_IN_RISE, E_IN_FALL]
    assert r.cell_glitches[0] == 4
    assert r.cell5[0, 1] == approx(sum(glitch_ratio(wi) * ei for wi, ei in zip(w, e)) / NORM, rel=1e-6)
    assert r.cell5[0, 0] == 0


def test_clock_pins_never_glitch():
    d = toy.build([toy.inv_cell()], [(0, [0, 1])], 2, period=1e-9, time_max=TMAX, clock_pins=[0])
    ev = toy.events(2, {0: [(0, 0), (3100, 1), (3150, 0)], 1: [(0, 1)]})
    r = run(d, ev)
    assert r.cell_glitches[0] == 0
    assert r.cell5[0, 0] == approx((E_IN_RISE + E_IN_FALL) / NORM, rel=1e-12)


def test_initial_event_is_never_a_glitch():
    d = inv_design()
    # no event at tick 0: the first event (index 0) is a real toggle from X
    # and is excluded from its period's glitch group
    ev = toy.events(2, {0: [(2100, 1), (2200, 0)], 1: [(0, 1)]})
    r = run(d, ev)
    # period 2 group = {event 1} only -> no glitch
    assert r.cell_glitches[0] == 0
    # X->1 counts half a toggle, 1->0 a full one
    assert r.cell_half_toggles[0] == 1 + 2
    e = 0.5 * E_IN_RISE + E_IN_FALL
    assert r.cell5[0, 0] == approx(e / NORM, rel=1e-12)


def test_unknown_and_high_impedance_values():
    d = inv_design()
    ev = toy.events(2, {0: [(0, 0), (2000, 2), (4000, 1), (6000, 3), (8000, 1)], 1: [(0, 1)]})
    r = run(d, ev)
    # 0->X: half toggle, n_rise 0.5 (rise); X->1: half, rise; 1->Z: full
    # toggle, fall (Z is value 3: not X, not a rise); Z->1: full toggle,
    # n_rise(3,1) = 0 -> fall
    e = 0.5 * E_IN_RISE + 0.5 * E_IN_RISE + E_IN_FALL + E_IN_FALL
    assert r.cell5[0, 0] == approx(e / NORM, rel=1e-12)
    assert r.cell_half_toggles[0] == 1 + 1 + 2 + 2
    # leakage: X and Z count as not-one -> !A
    lk = (f(2e-9) * 2000 + f(2e-9) * 2000 + f(1e-9) * 2000 + f(2e-9) * 2000 + f(1e-9) * 2000) / TMAX
    assert r.cell5[0, 4] == approx(lk, rel=1e-12)


def test_when_conditioned_input_tables_use_pre_event_state():
    d = toy.build([toy.nand_cell("N", when_tables=True)], [(0, [0, 1, 2])], 3, period=1e-9,
                  time_max=TMAX)
    # B=1 until 3000, then 0. A rises at 2000 (B=1 -> 7e-15), falls at 3000
    # together with B falling: both use the state before 3000 (B=1 -> 7e-15).
    # A rises again at 5000 (B=0 -> 5e-15). B's own fall costs 4e-15.
    ev = toy.events(3, {0: [(0, 0), (2000, 1), (3000, 0), (5000, 1)],
                        1: [(0, 1), (3000, 0)], 2: [(0, 1)]})
    r = run(d, ev)
    e = f(7e-15) + f(7e-15) + f(5e-15) + f(4e-15)
    assert r.cell5[0, 0] == approx(e / NORM, rel=1e-12)
    # leakage by the (A, B) bits: (s+1)*1e-9 for state index s = A + 2B
    lk = (f(3e-9) * 2000      # A=0,B=1 -> s=2
          + f(4e-9) * 1000    # A=1,B=1 -> s=3
          + f(1e-9) * 2000    # A=0,B=0 -> s=0
          + f(2e-9) * 5000)   # A=1,B=0 -> s=1
    assert r.cell5[0, 4] == approx(lk / TMAX, rel=1e-12)


def test_unconnected_pin_uses_default_state():
    d = toy.build([toy.inv_cell()], [(0, [-1, 1])], 2, period=1e-9, time_max=TMAX,
                  default_state=[1, 2])
    ev = toy.events(2, {1: [(0, 0)]})
    r = run(d, ev)
    assert r.cell5[0, 4] == approx(f(1e-9), rel=1e-12)


def test_group_totals_and_per_cycle_sums_agree():
    rng = np.random.default_rng(3)
    d, ev = toy.random_design(rng, n_cell=80, n_net=40, time_max=9_000, tpc=600)
    r = run(d, ev)
    # per-cell sums = totals; groups add up to totals
    v5 = np.stack([r.cell5[:, 4], r.cell5[:, 0] + r.cell5[:, 1], r.cell5[:, 1],
                   r.cell5[:, 2] + r.cell5[:, 3], r.cell5[:, 3]], axis=1)
    np.testing.assert_allclose(v5.sum(axis=0), r.totals, rtol=1e-12)
    np.testing.assert_allclose(r.groups.sum(axis=0), r.totals, rtol=1e-12)
    # energy conservation between per-cell and per-cycle views:
    # sum_c P_c * period = sum_cells E = P_cell * timeMax * ts
    np.testing.assert_allclose(r.cycle5[1].sum() * PF if False else r.cycle5[1].sum() * d.clk_period,
                               r.totals[1] * d.time_max * d.timescale, rtol=1e-6)
    np.testing.assert_allclose(r.cycle_events.sum(), r.cell_events.sum())
