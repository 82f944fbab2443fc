"""Builds the GCD design tape and its oracle results from the reference's
shipped example (test/gcd: sky130hd_tt.lib, gcd_sky130hd.v, .spef, .sdc and
the gcd_tb VCD, scope gcd_tb/gcd1, as test/gcd/power_vcd.tcl reads them).

Runs only where the reference tree is present; it writes
  tests/golden/gcd_tape.npz     design + events (the engine's inputs)
  tests/golden/gcd_oracle.npz   FP64 oracle outputs on that tape

The tape comes from gtpower_b200.sta_tape: slews, load caps and arc delays
from gtpower_b200.netlist's STA approximation, the clock and transitions
from the example's SDC (5 ns ideal clock on `clk`, 0.1 ns input
transition); the VCD binding follows ReadVcdActivities (nets first, then
instance pins, later bindings win).

Usage: python tests/golden/make_gcd_tape.py [/path/to/reference]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gtpower_b200 import sta_tape, tape  # noqa: E402


def build(ref_root: str):
    data = os.path.join(ref_root, "test", "gcd", "data")
    return sta_tape.build_tape(os.path.join(data, "sky130hd_tt.lib"), os.path.join(data, "gcd_sky130hd.v"),
                               os.path.join(data, "gcd_sky130hd.spef"), os.path.join(data, "gcd_sky130hd.sdc"),
                               os.path.join(data, "gcd_sky130hd.vcd"), "gcd_tb/gcd1")


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
