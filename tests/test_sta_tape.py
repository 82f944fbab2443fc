"""The design-tape producer (gtpower_b200.sta_tape): the SDC subset it reads,
and a tape built end to end from small hand-written Liberty, Verilog, SPEF,
SDC and VCD files, checked attribute by attribute and run through the
oracle."""
import numpy as np
import pytest

LIB = """
library (tiny) {
  time_unit : "1ns";
  voltage_unit : "1V";
  leakage_power_unit : "1nW";
  capacitive_load_unit (1, pf);
  default_operating_conditions : typ;
  operating_conditions (typ) { voltage : 1.5; }
  power_lut_template (p1) { variable_1 : input_transition_time; index_1 ("0.01, 1.0"); }
  power_lut_template (p2) { variable_1 : input_transition_time; variable_2 : total_output_net_capacitance;
                            index_1 ("0.01, 1.0"); index_2 ("0.001, 0.1"); }
  lu_table_template (d2) { variable_1 : input_transition_time; variable_2 : total_output_net_capacitance;
                           index_1 ("0.01, 1.0"); index_2 ("0.001, 0.1"); }
  cell (INVX) {
    cell_leakage_power : 2.0;
    leakage_power () { when : "A"; value : 1.0; }
    leakage_power () { when : "!A"; value : 3.0; }
    pin (A) {
      direction : input; capacitance : 0.002; rise_capacitance : 0.0024; fall_capacitance : 0.0018;
      internal_power () { rise_power (p1) { values ("0.001, 0.002"); } fall_power (p1) { values ("0.001, 0.003"); } }
    }
    pin (Y) {
      direction : output; function : "!A";
      internal_power () { related_pin : "A";
        rise_power (p2) { values ("0.01, 0.02", "0.03, 0.04"); }
        fall_power (p2) { values ("0.02, 0.03", "0.04, 0.05"); } }
      timing () { related_pin : "A"; timing_sense : negative_unate;
        cell_rise (d2) { values ("0.05, 0.5", "0.1, 0.6"); }
        cell_fall (d2) { values ("0.04, 0.4", "0.09, 0.5"); }
        rise_transition (d2) { values ("0.02, 0.8", "0.3, 1.0"); }
        fall_transition (d2) { values ("0.01, 0.6", "0.2, 0.9"); } }
    }
  }
  cell (CLKBUFX) {
    cell_leakage_power : 1.0;
    pin (A) { direction : input; capacitance : 0.003; }
    pin (X) {
      direction : output; function : "A";
      timing () { related_pin : "A"; timing_sense : positive_unate;
        cell_rise (d2) { values ("0.05, 0.5", "0.1, 0.6"); }
        cell_fall (d2) { values ("0.05, 0.5", "0.1, 0.6"); }
        rise_transition (d2) { values ("0.03, 0.7", "0.3, 1.0"); }
        fall_transition (d2) { values ("0.03, 0.7", "0.3, 1.0"); } }
    }
  }
  cell (DFFX) {
    cell_leakage_power : 5.0;
    ff (IQ, IQN) { next_state : "D"; clocked_on : "CLK"; }
    pin (D) { direction : input; capacitance : 0.0015; }
    pin (CLK) { direction : input; clock : true; capacitance : 0.0025;
      internal_power () { rise_power (p1) { values ("0.004, 0.005"); } fall_power (p1) { values ("0.003, 0.004"); } } }
    pin (Q) {
      direction : output; function : "IQ";
      internal_power () { related_pin : "CLK";
        rise_power (p2) { values ("0.02, 0.03", "0.04, 0.05"); }
        fall_power (p2) { values ("0.02, 0.03", "0.04, 0.05"); } }
      timing () { related_pin : "CLK"; timing_type : rising_edge;
        cell_rise (d2) { values ("0.2, 0.6", "0.3, 0.7"); }
        cell_fall (d2) { values ("0.2, 0.6", "0.3, 0.7"); }
        rise_transition (d2) { values ("0.05, 0.9", "0.2, 1.0"); }
        fall_transition (d2) { values ("0.04, 0.8", "0.2, 1.0"); } }
    }
  }
}
"""

VERILOG = """
module top (clk, a, y);
  input clk;
  input a;
  output y;
  wire n1, n2, clkb;
  INVX u1 (.A(a), .Y(n1));
  CLKBUFX cb (.A(clk), .X(clkb));
  DFFX r1 (.D(n1), .CLK(clkb), .Q(n2));
  INVX u2 (.A(n2), .Y(y));
endmodule
"""

SPEF = """*SPEF "IEEE 1481-1998"
*DESIGN "top"
*T_UNIT 1 PS
*C_UNIT 1 PF
*R_UNIT 1 OHM
*L_UNIT 1 HENRY
*D_NET n1 0.004
*END
*D_NET n2 0.005
*END
*D_NET clkb 0.010
*END
*D_NET y 0.002
*END
"""

SDC = """# clock, 4 ns
set per 4
create_clock -name core -period $per [get_ports clk]
set tr [expr $per * 0.05]
set_input_delay 1.0 -clock core [all_inputs]
set_input_transition $tr [all_inputs]
"""


def _vcd():
    rows = ["$timescale 1ps $end", "$scope module tb $end", "$scope module dut $end",
            "$var wire 1 ! clk $end", "$var wire 1 \" a $end", "$var wire 1 # n1 $end",
            "$var wire 1 $ n2 $end", "$var wire 1 % clkb $end", "$var wire 1 & y $end",
            "$upscope $end", "$upscope $end", "$enddefinitions $end", "#0",
            "0!", "0\"", "1#", "0$", "0%", "1&"]
    clk = 0
    a = 0
    q = 0
    for t in range(2000, 40001, 2000):          # clock edges every 2 ns (4 ns period)
        clk ^= 1
        rows.append(f"#{t}")
        rows.append(f"{clk}!")
        rows.append(f"{clk}%")
        if clk == 1:
            q = 1 - a                            # r1 samples n1 = !a
            rows.append(f"{q}$")
            rows.append(f"{1 - q}&")
        if t % 6000 == 0:
            rows.append(f"#{t + 700}")
            a ^= 1
            rows.append(f"{a}\"")
            rows.append(f"{1 - a}#")
    return "\n".join(rows) + "\n"


def _args(f):
    return f["lib"], f["v"], f["spef"], f["sdc"], f["vcd"], "tb/dut"


def _files(tmp_path, sdc=SDC):
    tmp_path.mkdir(parents=True, exist_ok=True)
    paths = {}
    for name, text in (("lib", LIB), ("v", VERILOG), ("spef", SPEF), ("sdc", sdc), ("vcd", _vcd())):
        p = tmp_path / f"top.{name}"
        p.write_text(text)
        paths[name] = str(p)
    return paths


def test_sdc_subset():
    from gtpower_b200.sta_tape import read_sdc
    text = """
    # comments and continuations
    set base 2.5
    set half [expr {$base / 2}]
    create_clock -name c0 -period [expr $base * 2] \\
        -waveform {0 ${half}} [get_ports {ck}]
    set_input_transition 0.2 [all_inputs]
    set_clock_transition [expr 0.01 + 0.02] [get_clocks c0]
    set_load 0.5 [all_outputs]
    """
    s = read_sdc(text, 1e-9)
    assert s.clock_port == "ck"
    assert s.period == pytest.approx(5e-9)
    assert s.input_transition == pytest.approx(0.2e-9)
    assert s.clock_transition == pytest.approx(0.03e-9)
    assert not s.propagated
    assert read_sdc(text + "\nset_propagated_clock [all_clocks]\n", 1e-9).propagated


def test_sdc_port_transitions_and_loads():
    from gtpower_b200.sta_tape import read_sdc
    s = read_sdc("set_input_transition 0.3 [get_ports {a b*}]\n"
                 "set_input_transition 0.1 [all_inputs]\n"
                 "set_input_transition 0.4 [get_ports a]\n"
                 "set_load 0.02 [all_outputs]\n", 1e-9)
    assert s.input_transition == pytest.approx(0.1e-9)
    assert s.port_transitions == [("a", pytest.approx(0.4e-9))]   # the [all_inputs] line replaced 0.3
    assert s.port_loads == [("__all_outputs__", 0.02)]


def test_tape_honours_port_transition_and_load(tmp_path):
    from gtpower_b200 import sta_tape
    base, _, _ = sta_tape.build_tape(*_args(_files(tmp_path / "a")))
    f = _files(tmp_path / "b", SDC + "set_input_transition 0.5 [get_ports a]\nset_load 0.03 [get_ports y]\n")
    d, _, _ = sta_tape.build_tape(*_args(f))
    k = {n: i for i, n in enumerate(d.cell_names)}
    u1_a = d.cell_pin_off[k["u1"]]
    u2_y = d.cell_pin_off[k["u2"]] + 1
    assert d.pin_slew_rise[u1_a] == pytest.approx(0.5e-9)
    assert d.pin_load_cap[u2_y] == pytest.approx(base.pin_load_cap[u2_y] + 0.03e-12, rel=1e-6)


def test_sdc_rejects_code():
    from gtpower_b200.sta_tape import read_sdc
    with pytest.raises(ValueError):
        read_sdc("set x [expr __import__('os')]", 1e-9)


def test_tape_from_files(tmp_path):
    from gtpower_b200 import sta_tape
    f = _files(tmp_path)
    d, ev, meta = sta_tape.build_tape(f["lib"], f["v"], f["spef"], f["sdc"], f["vcd"], "tb/dut")
    assert meta["clock_port"] == "clk" and meta["clock_period"] == pytest.approx(4e-9)
    assert meta["input_transition"] == pytest.approx(0.2e-9) and meta["ideal_clock"]
    assert d.n_cell == 4
    names = list(d.cell_names)
    k = {n: i for i, n in enumerate(names)}
    po = d.cell_pin_off

    def pin(cell, j):
        return po[k[cell]] + j

    # load caps: SPEF net cap + the larger of the load pins' rise and fall caps
    assert d.pin_load_cap[pin("u1", 1)] == pytest.approx((0.004 + 0.0015) * 1e-12, rel=1e-6)   # n1 -> r1.D
    assert d.pin_load_cap[pin("r1", 2)] == pytest.approx((0.005 + 0.0024) * 1e-12, rel=1e-6)   # n2 -> u2.A (rise cap)
    assert d.pin_load_cap[pin("cb", 1)] == pytest.approx((0.010 + 0.0025) * 1e-12, rel=1e-6)   # clkb -> r1.CLK
    # slews: primary inputs take the SDC transition; the ideal clock's network its transition (0)
    assert d.pin_slew_rise[pin("u1", 0)] == pytest.approx(0.2e-9)
    assert d.pin_slew_rise[pin("cb", 0)] == 0.0 and d.pin_slew_rise[pin("r1", 1)] == 0.0
    # report groups: the clock buffer is on the clock network, the flop sequential
    from gtpower_b200.design import GROUP_CLOCK, GROUP_COMBINATIONAL, GROUP_SEQUENTIAL
    assert d.cell_group[k["cb"]] == GROUP_CLOCK
    assert d.cell_group[k["r1"]] == GROUP_SEQUENTIAL
    assert d.cell_group[k["u1"]] == GROUP_COMBINATIONAL
    assert d.pin_is_clock[pin("r1", 1)] == 1
    # every pin is bound to a VCD signal; clk and clkb toggle every 2 ns
    assert meta["annotated_pins"] == d.n_pin
    assert ev.n_event > 40
    from oracle import oracle as orc
    r = orc.run(d, ev)
    assert r.totals[0] > 0 and r.totals[1] > 0 and r.totals[3] > 0
    assert int(r.cell_events.sum()) > 0


def test_propagated_clock_takes_buffer_slews(tmp_path):
    from gtpower_b200 import sta_tape
    f = _files(tmp_path, SDC + "set_propagated_clock [get_clocks core]\n")
    d, ev, meta = sta_tape.build_tape(f["lib"], f["v"], f["spef"], f["sdc"], f["vcd"], "tb/dut")
    assert not meta["ideal_clock"]
    k = {n: i for i, n in enumerate(d.cell_names)}
    clk_pin = d.cell_pin_off[k["r1"]] + 1
    assert d.pin_slew_rise[clk_pin] > 0.01e-9       # the buffer's rise_transition at its load


def test_gzipped_library(tmp_path):
    import gzip
    from gtpower_b200 import liberty
    p = tmp_path / "tiny.lib.gz"
    with gzip.open(p, "wt") as f:
        f.write(LIB)
    lib = liberty.read_library(str(p))
    assert sorted(lib.cells) == ["CLKBUFX", "DFFX", "INVX"]
    pins = lib.cell_data("INVX")["pins"]
    assert pins[0]["rise_capacitance"] == pytest.approx(0.0024e-12)
    assert pins[0]["fall_capacitance"] == pytest.approx(0.0018e-12)


def test_command_line(tmp_path):
    from gtpower_b200 import sta_tape, tape
    f = _files(tmp_path)
    out = tmp_path / "top_tape.npz"
    sta_tape.main(["--lib", f["lib"], "--verilog", f["v"], "--spef", f["spef"], "--sdc", f["sdc"],
                   "--vcd", f["vcd"], "--scope", "tb/dut", "--out", str(out)])
    d, ev, meta = tape.load(str(out))
    assert d.n_cell == 4 and meta["clock_port"] == "clk"
    assert np.all(np.diff(ev.net_off) >= 0)
