"""Builds the GCD design tape and its oracle results from the reference's
shipped example (test/gcd: sky130hd_tt.lib, gcd_sky130hd.v, .spef, .sdc and
the gcd_tb VCD, scope gcd_tb/gcd1, as test/gcd/power_vcd.tcl reads them).

Runs only where the reference tree is present; it writes
  tests/golden/gcd_tape.npz     design + events (the engine's inputs)
  tests/golden/gcd_oracle.npz   FP64 oracle outputs on that tape
  tests/golden/gcd_report.txt   report_power table from the oracle totals

Slews, load caps and arc delays come from gtpower_b200.netlist's STA
approximation (SDC: 5 ns clock on `clk`, 0.1 ns input transition); the VCD
binding follows ReadVcdActivities (nets first, then instance pins, later
bindings win).

Usage: python tests/golden/make_gcd_tape.py [/path/to/reference]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gtpower_b200 import liberty, netlist, tape, vcd  # noqa: E402
from gtpower_b200.design import Events  # noqa: E402


def build(ref_root: str):
    data = os.path.join(ref_root, "test", "gcd", "data")
    lib = liberty.read_library(os.path.join(data, "sky130hd_tt.lib"))
    mod = netlist.read_verilog(os.path.join(data, "gcd_sky130hd.v"))
    caps = netlist.read_spef_caps(os.path.join(data, "gcd_sky130hd.spef"))
    v = vcd.read(os.path.join(data, "gcd_sky130hd.vcd"))
    used = sorted({i.cell for i in mod.instances if i.cell in lib.cells})
    cells = {c: lib.cell_data(c) for c in used}
    d, info = netlist.build_design(mod, cells, caps, clock_port="clk", period=5e-9,
                                   input_slew=0.1e-9, timescale=v.timescale,
                                   time_max=v.time_max, voltage=lib.voltage, ideal_clock_slew=0.0)
    # bind waveforms: design nets, then instance pins (VCD order, later wins)
    nets = info["nets"]
    pin_index = {n: k for k, n in enumerate(info["pin_names"])}
    net_pins: dict[int, list[int]] = {}
    for q, n in enumerate(d.pin_net):
        if n >= 0:
            net_pins.setdefault(int(n), []).append(q)
    pin_bind: dict[int, tuple[str, int]] = {}
    for name, vid, bit in vcd.net_bindings(v, "gcd_tb/gcd1"):
        if name in nets:
            for q in net_pins.get(nets[name], []):
                pin_bind[q] = (vid, bit)
        elif name in pin_index:
            pin_bind[pin_index[name]] = (vid, bit)
    sources = sorted(set(pin_bind.values()))
    src_id = {s: k for k, s in enumerate(sources)}
    pin_net = np.full(d.n_pin, -1, np.int32)
    for q, s in pin_bind.items():
        pin_net[q] = src_id[s]
    off = [0]
    ts, vs = [], []
    for vid, bit in sources:
        t, val = vcd.bit_values(v, vid, bit)
        ts.append(t)
        vs.append(val)
        off.append(off[-1] + t.shape[0])
    ev = Events.from_values(np.asarray(off, np.int64),
                            np.concatenate(ts) if ts else np.zeros(0, np.int64),
                            np.concatenate(vs) if vs else np.zeros(0, np.uint8))
    d.pin_net = pin_net
    d.n_net = len(sources)
    meta = {"annotated_pins": len(pin_bind), "n_source": len(sources),
            "cells": len(d.cell_type), "time_max": v.time_max, "timescale": v.timescale}
    return d, ev, meta


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_gcd_tape.py <path of the reference checkout>")
    ref_root = sys.argv[1]
    d, ev, meta = build(ref_root)
    tape.save(os.path.join(HERE, "gcd_tape.npz"), d, ev, meta)
    from oracle import oracle as orc
    r = orc.run(d, ev)
    np.savez_compressed(os.path.join(HERE, "gcd_oracle.npz"), cell5=r.cell5, cycle5=r.cycle5,
                        totals=r.totals, groups=r.groups, cell_events=r.cell_events,
                        cell_glitches=r.cell_glitches, cell_half_toggles=r.cell_half_toggles,
                        cell_related=r.cell_related, cycle_events=r.cycle_events,
                        cycle_glitches=r.cycle_glitches)
    print(meta)
    print("totals (leak, int, g_int, sw, g_sw):", r.totals)
    print("n_period", d.n_period, "events", ev.n_event, "pin events", int(r.cell_events.sum()))


if __name__ == "__main__":
    main()
