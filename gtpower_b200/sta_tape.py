"""Design tapes for the power engine from a flat design's files, as
read_power_activities gets them in GTPower (test/gcd/power_vcd.tcl reads
Liberty, Verilog, SDC, SPEF and then the VCD of one testbench scope).

The per-pin attributes an STA run would give (slews, load caps, arc delays)
come from gtpower_b200.netlist's approximation; the clock, its period and
the transitions come from the SDC:

  - create_clock -period P [-name N] [-waveform {...}] PORT: the clock port
    and period;
  - set_input_transition T PORTS: the slew of primary inputs (all of them
    for [all_inputs], else the ports named, glob patterns allowed; later
    commands win);
  - set_load C PORTS: external load on top-level ports, added to their
    nets' load (in the library's capacitance unit);
  - set_clock_transition T CLOCKS: the ideal clock's transition (0 when
    unset), which every pin of an ideal clock's network takes;
  - set_propagated_clock: clock-network slews are propagated through the
    clock buffers instead.

SDC is Tcl; the reader evaluates the subset such constraint files use:
`set NAME VALUE`, `$NAME` and `${NAME}` substitution, `[expr ...]`
arithmetic, `[get_ports ...]`, `[get_clocks ...]`, `[all_inputs]`, `#`
comments and `\\` line continuations. Other commands are ignored. SDC times
are in the Liberty library's time unit, as OpenSTA reads them.

Command line:

    python -m gtpower_b200.sta_tape --lib L.lib --verilog D.v --spef D.spef \\
        --sdc D.sdc --vcd D.vcd --scope tb/dut --out D_tape.npz

The VCD binding follows ReadVcdActivities: design nets first, then instance
pins, in VCD order, later bindings winning.
"""
from __future__ import annotations

import argparse
import ast
import fnmatch
import operator
import re
from dataclasses import dataclass, field

import numpy as np

from . import liberty, netlist, tape, vcd
from .design import Design, Events


@dataclass
class Sdc:
    clock_port: str | None = None
    period: float | None = None          # s
    input_transition: float = 0.0        # s, for [all_inputs]
    clock_transition: float = 0.0        # s
    propagated: bool = False
    # (port pattern, value) in command order: transitions in s, loads in
    # library capacitance units
    port_transitions: list = field(default_factory=list)
    port_loads: list = field(default_factory=list)


_BINOPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul,
           ast.Div: operator.truediv, ast.Pow: operator.pow}
_UNOPS = {ast.UAdd: operator.pos, ast.USub: operator.neg}


def _arith(expr: str) -> float:
    """Value of a numeric expression of + - * / ** and parentheses."""
    def ev(n):
        if isinstance(n, ast.Expression):
            return ev(n.body)
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
            return float(n.value)
        if isinstance(n, ast.BinOp) and type(n.op) in _BINOPS:
            return _BINOPS[type(n.op)](ev(n.left), ev(n.right))
        if isinstance(n, ast.UnaryOp) and type(n.op) in _UNOPS:
            return _UNOPS[type(n.op)](ev(n.operand))
        raise ValueError(f"SDC expr: unsupported expression {expr!r}")
    return ev(ast.parse(expr.strip(), mode="eval"))


def _words(s: str) -> list[str]:
    """Tcl words: whitespace-separated, {...} kept as one word (braces removed)."""
    out, i = [], 0
    while i < len(s):
        if s[i].isspace():
            i += 1
            continue
        if s[i] == "{":
            depth, j = 1, i + 1
            while j < len(s) and depth:
                depth += {"{": 1, "}": -1}.get(s[j], 0)
                j += 1
            out.append(s[i + 1:j - 1])
            i = j
            continue
        j = i
        while j < len(s) and not s[j].isspace():
            j += 1
        out.append(s[i:j])
        i = j
    return out


def _substitute(cmd: str, vars_: dict[str, str]) -> str:
    def var(m):
        name = m.group(1) or m.group(2)
        if name not in vars_:
            raise ValueError(f"SDC: variable {name} is not set")
        return vars_[name]
    cmd = re.sub(r"\$\{(\w+)\}|\$(\w+)", var, cmd)
    # innermost brackets first
    while True:
        m = re.search(r"\[([^\[\]]*)\]", cmd)
        if not m:
            return cmd
        w = _words(m.group(1))
        if not w:
            val = ""
        elif w[0] == "expr":
            v = _arith(" ".join(w[1:]))
            val = repr(v)
        elif w[0] in ("get_ports", "get_pins", "get_nets", "get_clocks"):
            val = " ".join(x for x in w[1:] if not x.startswith("-"))
        elif w[0] == "all_inputs":
            val = "__all_inputs__"
        elif w[0] == "all_outputs":
            val = "__all_outputs__"
        else:
            val = ""
        cmd = cmd[:m.start()] + val + cmd[m.end():]


def read_sdc(text: str, time_unit: float) -> Sdc:
    """The clock and transition settings of an SDC file (times in seconds;
    time_unit = the Liberty library's time unit in seconds)."""
    sdc = Sdc()
    vars_: dict[str, str] = {}
    lines, buf = [], ""
    for raw in text.splitlines():
        line = raw.rstrip()
        if line.endswith("\\"):
            buf += line[:-1] + " "
            continue
        lines.append(buf + line)
        buf = ""
    if buf:
        lines.append(buf)
    for line in lines:
        s = line.strip()
        if not s or s.startswith("#"):
            continue
        w = _words(_substitute(s, vars_))
        if not w:
            continue
        cmd, args = w[0], w[1:]
        if cmd == "set" and len(args) >= 2:
            vars_[args[0]] = " ".join(args[1:])
        elif cmd == "create_clock":
            rest, k = [], 0
            while k < len(args):
                a = args[k]
                if a == "-period":
                    sdc.period = float(args[k + 1]) * time_unit
                    k += 2
                elif a in ("-name", "-waveform"):
                    k += 2
                elif a in ("-add",):
                    k += 1
                else:
                    rest.append(a)
                    k += 1
            ports = " ".join(rest).split()
            if ports and sdc.clock_port is None:
                sdc.clock_port = ports[0]
        elif cmd == "set_input_transition":
            vals = [a for a in args if not a.startswith("-")]
            if vals:
                v = float(vals[0]) * time_unit
                ports = " ".join(vals[1:]).split()
                if not ports or "__all_inputs__" in ports:
                    sdc.input_transition = v
                    sdc.port_transitions = []        # all inputs: earlier per-port values are replaced
                else:
                    sdc.port_transitions += [(pt, v) for pt in ports]
        elif cmd == "set_load":
            vals = [a for a in args if not a.startswith("-")]
            if len(vals) >= 2:
                sdc.port_loads += [(pt, float(vals[0])) for pt in " ".join(vals[1:]).split()]
        elif cmd == "set_clock_transition":
            vals = [a for a in args if not a.startswith("-")]
            if vals:
                sdc.clock_transition = float(vals[0]) * time_unit
        elif cmd == "set_propagated_clock":
            sdc.propagated = True
    return sdc


def build_tape(lib_path: str, verilog_path: str, spef_path: str | None, sdc_path: str, vcd_path: str,
               scope: str) -> tuple[Design, Events, dict]:
    """Design, events and a summary from a flat design's files. scope: the
    VCD scope of the design instance (e.g. "tb/dut")."""
    lib = liberty.read_library(lib_path)
    mod = netlist.read_verilog(verilog_path)
    caps = netlist.read_spef_caps(spef_path) if spef_path else {}
    v = vcd.read(vcd_path)
    with open(sdc_path) as f:
        sdc = read_sdc(f.read(), lib.time_scale)
    if sdc.clock_port is None or sdc.period is None:
        raise ValueError("the SDC defines no clock (create_clock -period ... PORT)")
    used = sorted({i.cell for i in mod.instances if i.cell in lib.cells})
    cells = {c: lib.cell_data(c) for c in used}
    input_slews = {}
    for pat, val in sdc.port_transitions:
        for port in mod.inputs:
            if fnmatch.fnmatchcase(port, pat):
                input_slews[port] = val
    port_loads: dict[str, float] = {}
    for pat, val in sdc.port_loads:
        ports = mod.outputs if pat == "__all_outputs__" else (
            mod.inputs if pat == "__all_inputs__" else
            [p for p in mod.inputs + mod.outputs if fnmatch.fnmatchcase(p, pat)])
        for port in ports:
            port_loads[port] = val * lib.cap_scale
    d, info = netlist.build_design(mod, cells, caps, clock_port=sdc.clock_port, period=sdc.period,
                                   input_slew=sdc.input_transition, timescale=v.timescale,
                                   time_max=v.time_max, voltage=lib.voltage,
                                   ideal_clock_slew=None if sdc.propagated else sdc.clock_transition,
                                   input_slews=input_slews, port_loads=port_loads)
    # bind waveforms: design nets, then instance pins (VCD order, later wins)
    nets = info["nets"]
    pin_index = {n: k for k, n in enumerate(info["pin_names"])}
    net_pins: dict[int, list[int]] = {}
    for q, n in enumerate(d.pin_net):
        if n >= 0:
            net_pins.setdefault(int(n), []).append(q)
    pin_bind: dict[int, tuple[str, int]] = {}
    for name, vid, bit in vcd.net_bindings(v, scope):
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
    meta = {"annotated_pins": len(pin_bind), "n_source": len(sources), "cells": len(d.cell_type),
            "time_max": v.time_max, "timescale": v.timescale, "clock_port": sdc.clock_port,
            "clock_period": sdc.period, "input_transition": sdc.input_transition,
            "ideal_clock": not sdc.propagated}
    return d, ev, meta


def main(argv: list[str] | None = None) -> None:
    ap = argparse.ArgumentParser(description="design tape for the B200 power engine")
    ap.add_argument("--lib", required=True)
    ap.add_argument("--verilog", required=True)
    ap.add_argument("--spef", default=None)
    ap.add_argument("--sdc", required=True)
    ap.add_argument("--vcd", required=True)
    ap.add_argument("--scope", required=True, help="VCD scope of the design instance, e.g. tb/dut")
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    d, ev, meta = build_tape(a.lib, a.verilog, a.spef, a.sdc, a.vcd, a.scope)
    tape.save(a.out, d, ev, meta)
    print(meta)


if __name__ == "__main__":
    main()
