"""Minimal Liberty reader for the power path.

Reads what the time-based power walk needs from a .lib file: units,
power/delay table templates, and per cell the pins (direction,
capacitance, clock flag), internal_power groups (related_pin, when,
rise_power/fall_power tables), leakage_power groups (when, value),
cell_leakage_power, timing groups (related_pin, timing_sense,
timing_type, cell_rise/cell_fall, rise_transition/fall_transition) and
whether the cell is sequential, a pad or a macro.

Units follow OpenSTA's LibertyReader (liberty/LibertyReader.cc:633-660,
766-878): table values of internal power are scaled by
voltage_unit^2 * capacitive_load_unit (energy), leakage by
leakage_power_unit, time axes by time_unit, capacitance axes and pin caps
by capacitive_load_unit.
"""
from __future__ import annotations

import json
import re
from dataclasses import dataclass, field
from typing import Any

# ---------------------------------------------------------------- parser

_TOKEN = re.compile(
    r'\s*(?:(/\*.*?\*/)|("(?:[^"\\]|\\.)*")|([{}();:,])|(\\\n)|([^\s{}();:,"]+))',
    re.S,
)


@dataclass
class Group:
    kind: str
    args: list[str]
    attrs: list[tuple[str, Any]] = field(default_factory=list)
    groups: list["Group"] = field(default_factory=list)

    def attr(self, name: str, default=None):
        for k, v in self.attrs:
            if k == name:
                return v
        return default

    def children(self, kind: str) -> list["Group"]:
        return [g for g in self.groups if g.kind == kind]


def _tokens(text: str):
    pos = 0
    n = len(text)
    while pos < n:
        m = _TOKEN.match(text, pos)
        if not m:
            if text[pos:].strip() == "":
                return
            raise ValueError(f"liberty: cannot tokenize at {pos}: {text[pos:pos + 40]!r}")
        pos = m.end()
        if m.group(1) or m.group(4):
            continue
        if m.group(2) is not None:
            yield ("str", m.group(2)[1:-1].replace("\\\n", ""))
        elif m.group(3) is not None:
            yield ("p", m.group(3))
        elif m.group(5) is not None:
            yield ("w", m.group(5))


def parse(text: str) -> Group:
    toks = list(_tokens(text))
    i = 0

    def parse_group_body(g: Group):
        nonlocal i
        while i < len(toks):
            t = toks[i]
            if t == ("p", "}"):
                i += 1
                return
            if t[0] not in ("w", "str"):
                i += 1
                continue
            name = t[1]
            i += 1
            if i < len(toks) and toks[i] == ("p", ":"):
                i += 1
                vals = []
                while i < len(toks) and toks[i] not in (("p", ";"), ("p", "}")):
                    vals.append(toks[i][1])
                    i += 1
                if i < len(toks) and toks[i] == ("p", ";"):
                    i += 1
                g.attrs.append((name, " ".join(vals)))
            elif i < len(toks) and toks[i] == ("p", "("):
                i += 1
                args = []
                cur = []
                while i < len(toks) and toks[i] != ("p", ")"):
                    if toks[i] == ("p", ","):
                        args.append(" ".join(cur))
                        cur = []
                    else:
                        cur.append(toks[i][1])
                    i += 1
                if cur:
                    args.append(" ".join(cur))
                i += 1  # ')'
                if i < len(toks) and toks[i] == ("p", "{"):
                    i += 1
                    sub = Group(name, args)
                    parse_group_body(sub)
                    g.groups.append(sub)
                else:
                    if i < len(toks) and toks[i] == ("p", ";"):
                        i += 1
                    g.attrs.append((name, args))
            else:
                # stray token
                continue

    root = Group("root", [])
    parse_group_body(root)
    return root


# ------------------------------------------------------- boolean `when`

class _Expr:
    """Boolean expression AST: ('port', name) | ('not', e) | ('and', a, b) |
    ('or', a, b) | ('xor', a, b) | ('one',) | ('zero',)."""


def parse_bool(expr: str):
    s = expr.replace('"', "").strip()
    toks = re.findall(r"[A-Za-z_][A-Za-z0-9_\[\]\.]*|[!'()&|*+^]|[01]", s)
    pos = 0

    def peek():
        return toks[pos] if pos < len(toks) else None

    def take():
        nonlocal pos
        t = toks[pos]
        pos += 1
        return t

    def p_or():
        a = p_xor()
        while peek() in ("|", "+"):
            take()
            a = ("or", a, p_xor())
        return a

    def p_xor():
        a = p_and()
        while peek() == "^":
            take()
            a = ("xor", a, p_and())
        return a

    def starts_primary(t):
        return t is not None and (t in ("!", "(", "0", "1") or re.match(r"[A-Za-z_]", t))

    def p_and():
        a = p_unary()
        while True:
            t = peek()
            if t in ("&", "*"):
                take()
                a = ("and", a, p_unary())
            elif starts_primary(t):  # juxtaposition = AND
                a = ("and", a, p_unary())
            else:
                return a

    def p_unary():
        if peek() == "!":
            take()
            return ("not", p_unary())
        e = p_primary()
        while peek() == "'":
            take()
            e = ("not", e)
        return e

    def p_primary():
        t = take()
        if t == "(":
            e = p_or()
            if peek() == ")":
                take()
            return e
        if t == "1":
            return ("one",)
        if t == "0":
            return ("zero",)
        return ("port", t)

    if not toks:
        return ("one",)
    return p_or()


def when_dnf(expr, pin_index: dict[str, int]) -> list[tuple[int, int]]:
    """General `when` -> DNF cubes (care, value) over pin bits. Used for
    internal power, matched by evalWhen (power/PowerUtils.cc:153-186)."""
    if expr is None:
        return [(0, 0)]
    names = sorted({n for n in _ports(expr)}, key=lambda n: pin_index[n])
    bits = [pin_index[n] for n in names]
    cubes = []
    # enumerate assignments of the referenced pins (few pins per cell)
    for m in range(1 << len(bits)):
        env = {names[k]: (m >> k) & 1 for k in range(len(bits))}
        if _eval(expr, env):
            care = 0
            val = 0
            for k, b in enumerate(bits):
                care |= 1 << b
                if env[names[k]]:
                    val |= 1 << b
            cubes.append((care, val))
    if not bits and _eval(expr, {}):
        return [(0, 0)]
    return cubes


def when_conjunction(expr, pin_index: dict[str, int]) -> list[tuple[int, int]]:
    """Leakage `when` -> one cube, following getWhenPinStates /
    collectWhenPinStates (power/PowerUtils.cc:110-151, 191-201): only
    conjunctions of literals (and negated disjunctions) are supported;
    anything else, or an unsatisfiable conjunction, matches no state."""
    if expr is None:
        return [(0, 0)]
    req: dict[int, int] = {}

    def collect(e, neg) -> bool:
        op = e[0]
        if op == "port":
            b = pin_index[e[1]]
            want = 0 if neg else 1
            if b in req and req[b] != want:
                return False
            req[b] = want
            return True
        if op == "not":
            return collect(e[1], not neg)
        if op == "one":
            return not neg
        if op == "zero":
            return neg
        if (op == "and" and not neg) or (op == "or" and neg):
            left = collect(e[1], neg)
            right = collect(e[2], neg)
            return left and right
        raise _Unsupported()

    try:
        ok = collect(expr, False)
    except _Unsupported:
        return []
    if not ok:
        return []
    care = 0
    val = 0
    for b, w in req.items():
        care |= 1 << b
        if w:
            val |= 1 << b
    return [(care, val)]


class _Unsupported(Exception):
    pass


def _ports(e):
    if e[0] == "port":
        yield e[1]
    for x in e[1:]:
        if isinstance(x, tuple):
            yield from _ports(x)


def _eval(e, env) -> bool:
    op = e[0]
    if op == "port":
        return bool(env[e[1]])
    if op == "not":
        return not _eval(e[1], env)
    if op == "and":
        return _eval(e[1], env) and _eval(e[2], env)
    if op == "or":
        return _eval(e[1], env) or _eval(e[2], env)
    if op == "xor":
        return _eval(e[1], env) != _eval(e[2], env)
    if op == "one":
        return True
    return False


# ------------------------------------------------------------ library

_UNIT = {"fs": 1e-15, "ps": 1e-12, "ns": 1e-9, "us": 1e-6, "ms": 1e-3, "s": 1.0,
         "ff": 1e-15, "pf": 1e-12, "nf": 1e-9, "uf": 1e-6,
         "pw": 1e-12, "nw": 1e-9, "uw": 1e-6, "mw": 1e-3, "w": 1.0,
         "mv": 1e-3, "v": 1.0}


def _unit_value(s: str) -> float:
    s = s.strip().strip('"').lower()
    m = re.match(r"([0-9.eE+-]*)\s*([a-z]+)", s)
    num = float(m.group(1)) if m.group(1) else 1.0
    return num * _UNIT[m.group(2)]


def _floats(s) -> list[float]:
    if isinstance(s, list):
        s = ",".join(s)
    return [float(x) for x in re.split(r"[,\s]+", s.replace('"', "").strip()) if x]


@dataclass
class Table:
    order: int
    axis_vars: list[str]            # "slew" | "cap"
    axes: list[list[float]]         # SI
    values: list[float]             # SI, row-major

    def to_json(self):
        return {"order": self.order, "axis_vars": self.axis_vars, "axes": self.axes,
                "values": self.values}


def _axis_var(v: str) -> str:
    v = v.strip('"')
    if v in ("input_transition_time", "input_net_transition", "related_pin_transition"):
        return "slew"
    if v in ("total_output_net_capacitance",):
        return "cap"
    return "other"


class Library:
    def __init__(self, root: Group):
        lib = root.groups[0]
        self.name = lib.args[0] if lib.args else ""
        self.time_scale = _unit_value(lib.attr("time_unit", "1ns"))
        cap = lib.attr("capacitive_load_unit", ["1", "pf"])
        self.cap_scale = float(cap[0]) * _UNIT[cap[1].strip('"').lower()]
        self.volt_scale = _unit_value(lib.attr("voltage_unit", "1V"))
        self.power_scale = _unit_value(lib.attr("leakage_power_unit", "1nW"))
        self.energy_scale = self.volt_scale * self.volt_scale * self.cap_scale
        self.voltage = 0.0
        opc = lib.attr("default_operating_conditions")
        for oc in lib.children("operating_conditions"):
            if opc is None or oc.args[0].strip('"') == str(opc).strip('"'):
                self.voltage = float(oc.attr("voltage", 0.0)) * self.volt_scale
        self.templates: dict[str, dict] = {}
        for kind in ("power_lut_template", "lu_table_template"):
            for t in lib.children(kind):
                d = {"vars": [], "index": []}
                for k in (1, 2, 3):
                    v = t.attr(f"variable_{k}")
                    if v is not None:
                        d["vars"].append(_axis_var(v))
                    idx = t.attr(f"index_{k}")
                    if idx is not None:
                        d["index"].append(_floats(idx))
                self.templates[t.args[0].strip('"')] = d
        self.cells = {c.args[0].strip('"'): c for c in lib.children("cell")}

    def _table(self, g: Group, value_scale: float) -> Table:
        tname = g.args[0].strip('"') if g.args else "scalar"
        tmpl = self.templates.get(tname, {"vars": [], "index": []})
        if tname == "scalar":
            return Table(0, [], [], [_floats(g.attr("values"))[0] * value_scale])
        vars_ = list(tmpl["vars"])
        axes = []
        for k in range(len(vars_)):
            idx = g.attr(f"index_{k + 1}")
            ax = _floats(idx) if idx is not None else list(tmpl["index"][k])
            scale = self.time_scale if vars_[k] == "slew" else self.cap_scale
            axes.append([a * scale for a in ax])
        vals = [v * value_scale for v in _floats(g.attr("values"))]
        return Table(len(vars_), vars_, axes, vals)

    def cell_data(self, name: str) -> dict:
        """Plain-data description of one cell (JSON-serialisable)."""
        c = self.cells[name]
        pins = []
        for p in c.children("pin"):
            pins.append(p)
        for b in c.children("bus"):
            pins.extend(b.children("pin"))
        inputs = [p for p in pins if p.attr("direction", "").strip('"') == "input"]
        outputs = [p for p in pins if p.attr("direction", "").strip('"') in ("output", "inout")]
        ordered = inputs + outputs
        names = [p.args[0].strip('"') for p in ordered]
        index = {n: i for i, n in enumerate(names)}
        out = {
            "name": name,
            "pins": [],
            "n_in": len(inputs),
            "internal_powers": [],
            "leakage_powers": [],
            "cell_leakage_power": None,
            "is_sequential": bool(c.children("ff") or c.children("latch") or c.children("statetable")
                                  or c.children("ff_bank") or c.children("latch_bank")),
            "is_pad": str(c.attr("pad_cell", "false")).strip('"') == "true",
            "is_macro": str(c.attr("is_macro_cell", "false")).strip('"') == "true",
            "timing": [],
            "functions": {},
        }
        clp = c.attr("cell_leakage_power")
        if clp is not None:
            out["cell_leakage_power"] = float(clp) * self.power_scale
        for p in ordered:
            pname = p.args[0].strip('"')
            capv = p.attr("capacitance")
            cap = float(capv) * self.cap_scale if capv is not None else 0.0
            # rise_capacitance / fall_capacitance override it per edge
            # (LibertyReader::visitRiseCap, visitFallCap)
            rcap, fcap = p.attr("rise_capacitance"), p.attr("fall_capacitance")
            out["pins"].append({
                "name": pname,
                "direction": p.attr("direction", "").strip('"'),
                "capacitance": cap,
                "rise_capacitance": float(rcap) * self.cap_scale if rcap is not None else cap,
                "fall_capacitance": float(fcap) * self.cap_scale if fcap is not None else cap,
                "clock": str(p.attr("clock", "false")).strip('"') == "true",
            })
            fn = p.attr("function")
            if fn is not None:
                out["functions"][pname] = fn.strip('"')
            for ip in p.children("internal_power"):
                rel = ip.attr("related_pin")
                rel_names = rel.strip('"').split() if rel else [None]
                when = ip.attr("when")
                expr = parse_bool(when) if when else None
                rise = ip.children("rise_power")
                fall = ip.children("fall_power")
                pw = ip.children("power")
                rt = self._table(rise[0], self.energy_scale).to_json() if rise else (
                    self._table(pw[0], self.energy_scale).to_json() if pw else None)
                ft = self._table(fall[0], self.energy_scale).to_json() if fall else (
                    self._table(pw[0], self.energy_scale).to_json() if pw else None)
                for rn in rel_names:
                    out["internal_powers"].append({
                        "pin": index[pname],
                        "related_pin": index[rn] if rn is not None and rn in index else -1,
                        "when": when_dnf(expr, index) if expr is not None else [[0, 0]],
                        "rise": rt,
                        "fall": ft,
                    })
            for tg in p.children("timing"):
                rel = tg.attr("related_pin")
                if not rel:
                    continue
                tt = str(tg.attr("timing_type", "combinational")).strip('"')
                sense = str(tg.attr("timing_sense", "non_unate")).strip('"')
                tabs = {}
                for k in ("cell_rise", "cell_fall", "rise_transition", "fall_transition"):
                    ch = tg.children(k)
                    if ch:
                        tabs[k] = self._table(ch[0], self.time_scale).to_json()
                for rn in rel.strip('"').split():
                    if rn not in index:
                        continue
                    out["timing"].append({"pin": index[pname], "related_pin": index[rn],
                                          "timing_type": tt, "timing_sense": sense,
                                          "tables": tabs})
        for lp in c.children("leakage_power"):
            when = lp.attr("when")
            expr = parse_bool(when) if when else None
            out["leakage_powers"].append({
                "when": when_conjunction(expr, index),
                "power": float(lp.attr("value")) * self.power_scale,
            })
        return out


def read_library(path: str) -> Library:
    """A Liberty file, plain or gzip-compressed (.gz)."""
    if path.endswith(".gz"):
        import gzip
        with gzip.open(path, "rt") as f:
            return Library(parse(f.read()))
    with open(path) as f:
        return Library(parse(f.read()))


def extract(path: str, cells: list[str], out_json: str) -> None:
    """Writes the plain-data description of `cells` to a JSON file."""
    lib = read_library(path)
    data = {"library": lib.name, "voltage": lib.voltage,
            "cells": {n: lib.cell_data(n) for n in cells}}
    with open(out_json, "w") as f:
        json.dump(data, f, separators=(",", ":"))


def load_json(path: str) -> dict:
    with open(path) as f:
        return json.load(f)
