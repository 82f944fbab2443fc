"""The reference's shipped GCD example (test/gcd, power_vcd.tcl).

tests/golden/gcd_tape.npz is the design tape built from the example's
Liberty, Verilog, SPEF, SDC and VCD by tests/golden/make_gcd_tape.py;
tests/golden/gcd_oracle.npz holds the FP64 oracle's outputs on it.

The reference's own golden for this run is the report_power table of
test/power_vcd.ok (3 significant digits). Its leakage depends only on the
VCD states and Liberty leakage tables, so the oracle must reproduce it
closely; internal and switching power also depend on slews and load caps,
which the tape takes from an STA approximation, so they match less tightly.
The example's SDC defines an ideal clock (no propagated clock), so every
clock-network pin takes the clock's ideal transition, 0, as OpenSTA gives
it; with propagated clock-buffer slews internal power was 2-3% low.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TAPE = os.path.join(HERE, "golden", "gcd_tape.npz")
GOLD = os.path.join(HERE, "golden", "gcd_oracle.npz")

# test/power_vcd.ok: group -> (internal, switching, leakage, total) W
POWER_VCD_OK = {
    "Sequential": (3.05e-04, 3.85e-05, 2.92e-10, 3.44e-04),
    "Combinational": (9.90e-05, 1.59e-04, 6.76e-10, 2.58e-04),
    "Clock": (4.82e-05, 1.20e-04, 2.30e-11, 1.69e-04),
    "Total": (4.53e-04, 3.18e-04, 9.91e-10, 7.71e-04),
}
GROUP_INDEX = {"Combinational": 0, "Sequential": 1, "Clock": 2}


def load():
    from gtpower_b200 import tape
    return tape.load(TAPE)


def test_tape_matches_reference_annotation_count():
    d, ev, meta = load()
    # "Annotated 937 pin activities" in power_vcd.ok counts the 54 top-level
    # port pins (clk, req_*, resp_*, 32 req_msg, 16 resp_msg) and 883 cell pins
    assert meta["annotated_pins"] + 54 == 937
    assert d.n_cell == 252
    assert d.ticks_per_cycle == 5000 and d.n_period == 26


def test_oracle_reproduces_committed_golden():
    from oracle import oracle as orc
    d, ev, _ = load()
    r = orc.run(d, ev)
    g = np.load(GOLD)
    np.testing.assert_allclose(r.cell5, g["cell5"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(r.cycle5, g["cycle5"], rtol=1e-12, atol=0)
    for k in ("cell_events", "cell_glitches", "cell_half_toggles", "cell_related",
              "cycle_events", "cycle_glitches"):
        assert np.array_equal(getattr(r, k), g[k]), k


@pytest.mark.parametrize("group", ["Sequential", "Combinational", "Clock", "Total"])
def test_oracle_against_reference_report(group):
    from oracle import oracle as orc
    d, ev, _ = load()
    r = orc.run(d, ev)
    if group == "Total":
        v = r.totals
    else:
        v = r.groups[GROUP_INDEX[group]]
    internal, switching, leakage = v[1], v[3], v[0]
    ok_int, ok_sw, ok_leak, ok_tot = POWER_VCD_OK[group]
    assert leakage == pytest.approx(ok_leak, rel=0.015)         # state-only: within 1.5%
    assert internal == pytest.approx(ok_int, rel=0.01)          # slew-dependent: within 1%
    assert switching == pytest.approx(ok_sw, rel=0.05)          # load-cap-dependent: within 5%
    assert internal + switching + leakage == pytest.approx(ok_tot, rel=0.015)


def test_report_power_table_layout(tmp_path):
    """B200Power.report_power formats the group table as Power.tcl does;
    checked here on the oracle's numbers through the same formatter."""
    from gtpower_b200.power import B200Power, Results
    d, ev, _ = load()
    from oracle import oracle as orc
    r = orc.run(d, ev)
    eng = B200Power.__new__(B200Power)          # formatter only, no device
    eng.design = d
    eng._results = Results(r.cell5.astype(np.float32), r.cycle5.astype(np.float32), r.totals, r.groups)
    eng.n_period = d.n_period
    eng.ctx = None
    text = eng.report_power()
    lines = text.splitlines()
    assert lines[0].split() == ["Group", "Internal", "Switching", "Leakage", "Total"]
    assert lines[2] == "-" * 64
    assert [l.split()[0] for l in lines[3:8]] == ["Sequential", "Combinational", "Clock", "Macro", "Pad"]
    assert lines[-2].startswith("Total")
    eng.print_cell_res(str(tmp_path / "cuda_cell_power.txt"))
    rows = (tmp_path / "cuda_cell_power.txt").read_text().splitlines()
    assert rows[0].split("\t") == ["cell", "Internal_Power", "Glitch_Internal_Power", "Switching_Power",
                                   "Glitch_Switching_Power", "Leakage_Power", "Total_Power", "Standard_Cell"]
    assert len(rows) == d.n_cell + 1


def test_vcd_reader_semantics(tmp_path):
    from gtpower_b200 import vcd
    text = """$timescale 1ps $end
$scope module tb $end
$scope module dut $end
$var wire 1 ! a $end
$var wire 4 " bus [3:0] $end
$var wire 1 # b $end
$upscope $end
$upscope $end
$enddefinitions $end
#0
$dumpvars
1!
b0101 "
$end
#10
1!
0!
b0111 "
#20
x!
bx1 "
1#
#30
u!
"""
    p = tmp_path / "t.vcd"
    p.write_text(text)
    v = vcd.read(str(p))
    assert v.timescale == 1e-12 and v.time_max == 30
    a_id = [x.id for x in v.vars if x.name.endswith("/a")][0]
    t, val = vcd.bit_values(v, a_id, 0)
    # repeated 1 at #10 dropped; X and U kept (U read as X)
    assert t.tolist() == [0, 10, 20, 30] and val.tolist() == [1, 0, 2, 2]
    b_id = [x.id for x in v.vars if x.name.endswith("/b")][0]
    t, val = vcd.bit_values(v, b_id, 0)
    # first change at #20: an initial X is inserted at tick 0
    assert t.tolist() == [0, 20] and val.tolist() == [2, 1]
    bus_id = [x.id for x in v.vars if "bus" in x.name][0]
    # bit 1 of 0101, 0111, 0 (bx1 -> 0): per-bit repeats survive
    t, val = vcd.bit_values(v, bus_id, 1)
    assert t.tolist() == [0, 10, 20] and val.tolist() == [0, 1, 0]
    binds = vcd.net_bindings(v, "tb/dut")
    names = [b[0] for b in binds]
    assert "bus[0]" in names and "bus[3]" in names
    assert dict((n, bit) for n, _, bit in binds)["bus[0]"] == 0   # bit `to` is the LSB


@pytest.mark.gpu
def test_engine_on_gcd_tape():
    from gtpower_b200 import B200Power
    from oracle import oracle as orc
    from tests.parity import compare
    d, ev, _ = load()
    with B200Power(d, collect_counts=True) as eng:
        eng.read_power_activities(ev)
        res = eng.fetch(counts=True)
    compare(res, orc.run(d, ev))
