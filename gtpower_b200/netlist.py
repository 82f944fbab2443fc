"""Flat gate-level netlist ingest for the power engine.

Reads a flat structural Verilog module (cell instances with named port
connections), lumped net capacitance from SPEF (*D_NET totals), and builds
a `Design` with the per-pin quantities an STA run would provide:

  - load cap of an output pin = SPEF total cap of its net + the Liberty
    capacitance of the net's load pins, for the rise and the fall edge
    (rise_capacitance / fall_capacitance where the library gives them),
    the larger of the two (GraphDelayCalc::loadCap with lumped parasitics);
  - slews: primary inputs take the SDC input transition; each driver
    output takes the worst rise_transition / fall_transition of its delay
    arcs at (worst input slew, load cap), propagated in topological order;
    every pin on a net takes the net's slew (no wire degradation);
  - arc delays: cell_rise / cell_fall at (input pin slew, load cap) for the
    edges the arc's timing_sense / timing_type allows;
  - report groups as Power::power classifies instances (power/Power.cc:
    338-347): macro, pad, clock network (every output is a clock pin, i.e.
    on the clock's buffer tree), sequential, combinational.

This is an STA approximation (OpenSTA's delay calculation also models wire
RC and slew degradation); it is the documented source of the slews, caps
and delays on the GCD tape.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

import numpy as np

from .design import (CellLibrary, Design, GROUP_CLOCK, GROUP_COMBINATIONAL, GROUP_MACRO,
                     GROUP_PAD, GROUP_SEQUENTIAL)
from .synth import _arc_edges, _interp2
from .vcd import normalize

_ID = r"(?:\\\S+\s|[A-Za-z_][\w$]*)"


@dataclass
class Instance:
    name: str
    cell: str
    conns: dict[str, str]


@dataclass
class Module:
    name: str
    inputs: list[str] = field(default_factory=list)
    outputs: list[str] = field(default_factory=list)
    instances: list[Instance] = field(default_factory=list)


def _expand_ports(decl: str, width: str | None) -> list[str]:
    names = [normalize(x) for x in decl.split(",") if x.strip()]
    if not width:
        return names
    m = re.match(r"\[(\d+):(\d+)\]", width)
    hi, lo = int(m.group(1)), int(m.group(2))
    rng = range(lo, hi + 1) if hi >= lo else range(hi, lo + 1)
    return [f"{n}[{b}]" for n in names for b in rng]


def read_verilog(path: str) -> Module:
    text = open(path).read()
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    m = re.search(r"module\s+(\S+)\s*\(", text)
    mod = Module(m.group(1))
    body = text[m.end():]
    for kind, width, decl in re.findall(r"\b(input|output)\s*(\[\d+:\d+\])?\s*([^;]+);", body):
        (mod.inputs if kind == "input" else mod.outputs).extend(_expand_ports(decl, width))
    inst_re = re.compile(r"\b(\w+)\s+(" + _ID + r")\s*\((.*?)\)\s*;", re.S)
    for cell, name, conns in inst_re.findall(body):
        if cell in ("module", "input", "output", "wire", "assign"):
            continue
        cm = {}
        for pin, net in re.findall(r"\.(\w+)\s*\(\s*([^()]*?)\s*\)", conns):
            if net:
                cm[pin] = normalize(net)
        mod.instances.append(Instance(normalize(name), cell, cm))
    return mod


def _spef_name(s: str) -> str:
    """A SPEF name as the netlist spells it: SPEF escapes '.', '[', ']', '$'
    and the like with a backslash (dpath\\.a\\[0\\] for dpath.a[0])."""
    return normalize(re.sub(r"\\(.)", r"\1", s))


def read_spef_caps(path: str) -> dict[str, float]:
    """Net name -> total capacitance in farads."""
    caps = {}
    name_map = {}
    c_unit = 1e-12
    in_map = False
    with open(path) as f:
        for line in f:
            s = line.strip()
            if s.startswith("*C_UNIT"):
                p = s.split()
                c_unit = float(p[1]) * {"PF": 1e-12, "FF": 1e-15, "NF": 1e-9}[p[2].upper()]
            elif s.startswith("*NAME_MAP"):
                in_map = True
            elif in_map and s.startswith("*") and not s.startswith("*D_NET") and " " in s:
                k, v = s.split(None, 1)
                if k[1:].isdigit():
                    name_map[k] = _spef_name(v)
                else:
                    in_map = False
            if s.startswith("*D_NET"):
                in_map = False
                _, ref, cap = s.split()[:3]
                caps[name_map.get(ref, _spef_name(ref))] = float(cap) * c_unit
    return caps


def build_design(mod: Module, cells: dict, spef_caps: dict[str, float], *, clock_port: str,
                 period: float, input_slew: float, timescale: float, time_max: int,
                 voltage: float, ideal_clock_slew: float | None = None,
                 input_slews: dict[str, float] | None = None,
                 port_loads: dict[str, float] | None = None) -> tuple[Design, dict]:
    """Design for the instances whose cell has Liberty data (others are
    black boxes the power walk skips, as the reference does).
    ideal_clock_slew: the slew of every clock-network net when the clock is
    ideal (OpenSTA's clock transition, set_clock_transition, 0 by default);
    None propagates the clock buffers' slews like any other net.
    input_slews: per-port slews (s) that replace input_slew for those ports;
    port_loads: external load (F) on top-level ports (SDC set_load), added
    to the load of the port's net."""
    insts = [i for i in mod.instances if i.cell in cells]
    used = sorted({i.cell for i in insts})
    lib = CellLibrary([cells[c] for c in used])
    tindex = {c: k for k, c in enumerate(used)}
    nets: dict[str, int] = {}

    def nid(n):
        if n not in nets:
            nets[n] = len(nets)
        return nets[n]

    for p in mod.inputs + mod.outputs:
        nid(p)
    cell_type, pin_off, pin_net, pin_names = [], [0], [], []
    for inst in insts:
        c = cells[inst.cell]
        cell_type.append(tindex[inst.cell])
        for p in c["pins"]:
            n = inst.conns.get(p["name"])
            pin_net.append(nid(n) if n is not None else -1)
            pin_names.append(f"{inst.name}/{p['name']}")
        pin_off.append(len(pin_net))
    n_net = len(nets)
    cell_type = np.asarray(cell_type, np.int32)
    pin_off = np.asarray(pin_off, np.int32)
    pin_net = np.asarray(pin_net, np.int32)
    n_pin = pin_net.shape[0]

    # driver of each net and load caps
    is_out = np.zeros(n_pin, bool)
    pin_cap = np.zeros((2, n_pin))        # rise, fall
    pin_clock_attr = np.zeros(n_pin, np.uint8)
    for k, inst in enumerate(insts):
        c = cells[inst.cell]
        for j, p in enumerate(c["pins"]):
            q = pin_off[k] + j
            is_out[q] = j >= c["n_in"]
            pin_cap[0, q] = p.get("rise_capacitance", p["capacitance"])
            pin_cap[1, q] = p.get("fall_capacitance", p["capacitance"])
            pin_clock_attr[q] = 1 if p["clock"] else 0
    net_cap = np.zeros(n_net)
    for name, n in nets.items():
        net_cap[n] = spef_caps.get(name, 0.0)
    # the larger of the rise and fall loads (wire + the load pins' caps of
    # that edge), as GraphDelayCalc::loadCap takes over both edges
    valid = pin_net >= 0
    ld = valid & ~is_out
    load_rf = np.stack([net_cap.copy(), net_cap.copy()])
    for e in range(2):
        np.add.at(load_rf[e], pin_net[ld], pin_cap[e, ld])
    for port, c_ext in (port_loads or {}).items():
        if port in nets:
            load_rf[:, nets[port]] += c_ext
    load = np.maximum(load_rf[0], load_rf[1])
    driver = np.full(n_net, -1, np.int64)
    for q in np.nonzero(valid & is_out)[0]:
        driver[pin_net[q]] = q
    pin_cell = np.repeat(np.arange(len(insts)), np.diff(pin_off))

    # clock network: nets reached from the clock port through combinational cells
    clock_nets = {nets[clock_port]} if clock_port in nets else set()
    changed = True
    while changed:
        changed = False
        for k, inst in enumerate(insts):
            c = cells[inst.cell]
            if c["is_sequential"]:
                continue
            ins = [pin_net[pin_off[k] + j] for j in range(c["n_in"])]
            outs = [pin_net[pin_off[k] + j] for j in range(c["n_in"], len(c["pins"]))]
            if any(m in clock_nets for m in ins):
                for m in outs:
                    if m >= 0 and m not in clock_nets:
                        clock_nets.add(m)
                        changed = True
    # slews in topological order over combinational arcs; with an ideal clock
    # (no propagated clock in the SDC) every clock-network net takes the
    # clock's ideal transition, as OpenSTA gives an ideal clock's pins
    net_slew = np.full((2, n_net), np.nan)
    for p in mod.inputs:
        net_slew[:, nets[p]] = (input_slews or {}).get(p, input_slew)
    if ideal_clock_slew is not None:
        for m in clock_nets:
            net_slew[:, m] = ideal_clock_slew
    resolved = ~np.isnan(net_slew[0])
    pending = set(np.nonzero(driver >= 0)[0].tolist())
    if ideal_clock_slew is not None:
        pending -= clock_nets
    for _ in range(len(insts) + 2):
        progressed = False
        for n in list(pending):
            q = driver[n]
            k = pin_cell[q]
            c = cells[insts[k].cell]
            j = q - pin_off[k]
            arcs = [tg for tg in c["timing"] if tg["pin"] == j and _arc_edges(tg["timing_type"], tg["timing_sense"])]
            ins = [pin_off[k] + tg["related_pin"] for tg in arcs]
            in_nets = [pin_net[x] for x in ins if pin_net[x] >= 0]
            seq = any(tg["timing_type"] in ("rising_edge", "falling_edge") for tg in arcs)
            if not seq and any(not resolved[m] for m in in_nets):
                continue
            r = f = 0.0
            for tg, x in zip(arcs, ins):
                m = pin_net[x]
                s_in = max(net_slew[0, m], net_slew[1, m]) if m >= 0 and resolved[m] else input_slew
                tabs = tg["tables"]
                if "rise_transition" in tabs:
                    r = max(r, float(_interp2(tabs["rise_transition"], np.asarray([s_in]), np.asarray([load[n]]))[0]))
                if "fall_transition" in tabs:
                    f = max(f, float(_interp2(tabs["fall_transition"], np.asarray([s_in]), np.asarray([load[n]]))[0]))
            net_slew[0, n] = r if r > 0 else input_slew
            net_slew[1, n] = f if f > 0 else input_slew
            resolved[n] = True
            pending.discard(n)
            progressed = True
        if not pending or not progressed:
            break
    for n in pending:  # combinational loops: fall back to the input slew
        net_slew[:, n] = input_slew
    net_slew[np.isnan(net_slew)] = input_slew
    slew_r = np.where(valid, net_slew[0, np.maximum(pin_net, 0)], input_slew).astype(np.float32)
    slew_f = np.where(valid, net_slew[1, np.maximum(pin_net, 0)], input_slew).astype(np.float32)
    pin_load = np.where(is_out & valid, load[np.maximum(pin_net, 0)], 0.0).astype(np.float32)

    # arc delays
    arc_off = np.zeros(len(insts), np.int64)
    total = 0
    for k, inst in enumerate(insts):
        c = cells[inst.cell]
        arc_off[k] = total
        total += 4 * c["n_in"] * (len(c["pins"]) - c["n_in"])
    arc = np.full(max(total, 1), np.nan, np.float32)
    for k, inst in enumerate(insts):
        c = cells[inst.cell]
        n_in = c["n_in"]
        for tg in c["timing"]:
            o = tg["pin"] - n_in
            qq = tg["related_pin"]
            if o < 0 or qq >= n_in:
                continue
            for fr, to in _arc_edges(tg["timing_type"], tg["timing_sense"]):
                tab = tg["tables"].get("cell_rise" if to == 0 else "cell_fall")
                if tab is None:
                    continue
                s = slew_r[pin_off[k] + qq] if fr == 0 else slew_f[pin_off[k] + qq]
                dl = _interp2(tab, np.asarray([float(s)]), np.asarray([float(pin_load[pin_off[k] + n_in + o])]))[0]
                arc[arc_off[k] + (o * n_in + qq) * 4 + 2 * fr + to] = np.float32(dl)

    group = np.zeros(len(insts), np.uint8)
    for k, inst in enumerate(insts):
        c = cells[inst.cell]
        outs = [pin_net[pin_off[k] + j] for j in range(c["n_in"], len(c["pins"]))]
        if c["is_macro"]:
            group[k] = GROUP_MACRO
        elif c["is_pad"]:
            group[k] = GROUP_PAD
        elif outs and all(m in clock_nets for m in outs):
            group[k] = GROUP_CLOCK
        elif c["is_sequential"]:
            group[k] = GROUP_SEQUENTIAL
        else:
            group[k] = GROUP_COMBINATIONAL
    d = Design(lib=lib, timescale=timescale, clk_period=float(np.float32(period)), time_max=time_max,
               n_net=n_net, cell_type=cell_type, cell_pin_off=pin_off, cell_group=group,
               cell_arc_off=arc_off, pin_net=pin_net, pin_slew_rise=slew_r, pin_slew_fall=slew_f,
               pin_load_cap=pin_load, pin_voltage=np.full(n_pin, voltage, np.float32),
               pin_default_state=np.full(n_pin, 2, np.uint8), pin_is_clock=pin_clock_attr,
               arc_delay=arc, cell_names=[i.name for i in insts], top_name=mod.name)
    return d, {"nets": nets, "pin_names": pin_names}
