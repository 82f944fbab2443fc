"""VCD reader with the reference's value semantics, and per-net event lists.

Follows power/VcdReader.cc and power/Vcd.cc:
  - values are upper-cased; scalar 0/1/X/U/Z changes are stored
    (VcdReader::parseVarValues, VcdReader.cc:247-301);
  - a vector value `b...` whose first digit is x/u/z becomes bus value 0;
    otherwise the leading binary digits are read (strtol base 2, which
    saturates at 2^63 - 1);
  - real values are skipped;
  - a change equal to the previous value of the same id is dropped, and an
    initial value is inserted at tick 0 when the first change is later
    ('X' for scalars, bus value 0 for vectors) (Vcd::varAppendValue /
    varAppendBusValue, Vcd.cc:204-234);
  - bit b of a vector value is ((bus_value >> b) & 1) (VcdValue::value,
    Vcd.cc:271-277), so per-bit repeats survive as events;
  - time_max is the last timestamp; the timescale is value * unit.
Per-net event lists map each net (or instance pin) named in the VCD below
`scope` to its var and bit as ReadVcdActivities does
(power/ReadVcdActivities.cc:510-619): a vector `name[from:to]` gives bit
`to` the LSB of the value.
"""
from __future__ import annotations

import gzip
import re
from dataclasses import dataclass, field

import numpy as np

_UNIT = {"fs": 1e-15, "ps": 1e-12, "ns": 1e-9, "us": 1e-6, "ms": 1e-3, "s": 1.0}
VALUE_CODE = {"0": 0, "1": 1, "X": 2, "Z": 3, "U": 2}   # U: the reference CPU path throws; mapped to X


@dataclass
class VcdVar:
    name: str          # full hierarchical name with '/' separators
    width: int
    id: str
    type: str


@dataclass
class Vcd:
    timescale: float = 1.0
    time_max: int = 0
    vars: list = field(default_factory=list)
    # id -> (times list, chars list | None, bus list | None, width)
    values: dict = field(default_factory=dict)


def _open(path):
    return gzip.open(path, "rt") if path.endswith(".gz") else open(path)


def read(path: str) -> Vcd:
    with _open(path) as f:
        return read_text(f.read())


def split_header(raw: bytes) -> tuple[bytes, bytes]:
    """(header, body) of a VCD file's bytes: the body starts after the
    `$end` that closes `$enddefinitions`."""
    m = re.search(rb"(?:^|\s)\$enddefinitions(?=\s|$)", raw)
    if not m:
        return raw, b""
    e = re.search(rb"(?:^|\s)\$end(?=\s|$)", raw[m.end():])
    if not e:
        return raw, b""
    cut = m.end() + e.end()
    return raw[:cut], raw[cut:]


def read_text(text: str) -> Vcd:
    v = Vcd()
    toks = text.split()
    n = len(toks)
    i = 0
    scope: list[str] = []
    widths: dict[str, int] = {}
    time = 0
    body = False

    def stmt():
        nonlocal i
        out = []
        while i < n and toks[i] != "$end":
            out.append(toks[i])
            i += 1
        i += 1
        return out

    while i < n:
        t = toks[i]
        i += 1
        if not body:
            if t == "$timescale":
                s = stmt()
                txt = "".join(s)
                m = re.match(r"([0-9.]+)\s*([a-z]+)", txt)
                v.timescale = float(m.group(1)) * _UNIT[m.group(2)]
            elif t == "$var":
                s = stmt()
                if len(s) in (4, 5):
                    name = "/".join(scope + [s[3].replace("/", "\\/")])
                    if len(s) == 5:
                        if name.startswith("\\"):
                            name += " "
                        name += s[4]
                    var = VcdVar(name, int(s[1]), s[2], s[0])
                    v.vars.append(var)
                    widths.setdefault(var.id, var.width)
                    v.values.setdefault(var.id, ([], [], [], var.width))
            elif t == "$scope":
                s = stmt()
                scope.append(s[1])
            elif t == "$upscope":
                stmt()
                scope.pop()
            elif t in ("$date", "$comment", "$version"):
                stmt()
            elif t == "$enddefinitions":
                stmt()
                body = True
            continue
        c0 = t[0].upper()
        if c0 == "#" and len(t) > 1:
            time = int(t[1:])
        elif c0 in "01XUZ" and len(t) > 1:
            vid = t[1:]
            ts, cs, bs, w = v.values[vid]
            if not cs or cs[-1] != c0:
                if not ts and time != 0:
                    ts.append(0); cs.append("X"); bs.append(0)
                ts.append(time); cs.append(c0); bs.append(0)
        elif c0 == "B":
            vid = toks[i]
            i += 1
            c1 = t[1].upper() if len(t) > 1 else "0"
            if c1 in "XUZ":
                bus = 0
            else:
                # the leading binary digits, as strtol reads them (saturated
                # at its largest value)
                m = re.match(r"[01]*", t[1:])
                bus = min(int(m.group(0), 2), (1 << 63) - 1) if m.group(0) else 0
            ts, cs, bs, w = v.values[vid]
            if not bs or bs[-1] != bus or not ts:
                if not ts and time != 0:
                    ts.append(0); cs.append(None); bs.append(0)
                ts.append(time); cs.append(None); bs.append(bus)
        elif c0 == "R":
            i += 1  # real value: id follows
        # '$dumpvars', '$end', ... : nothing
    v.time_max = time
    return v


def bit_values(v: Vcd, vid: str, bit: int) -> tuple[np.ndarray, np.ndarray]:
    ts, cs, bs, w = v.values[vid]
    times = np.asarray(ts, dtype=np.int64)
    vals = np.empty(len(ts), dtype=np.uint8)
    for k in range(len(ts)):
        c = cs[k]
        vals[k] = ((bs[k] >> bit) & 1) if c is None else VALUE_CODE[c]
    return times, vals


_BUS = re.compile(r"^(.*)\[(\d+):(\d+)\]$")


def net_bindings(v: Vcd, scope: str) -> list[tuple[str, str, int]]:
    """(design name, var id, bit) for every wire/reg var below `scope`, in
    VCD order; a later binding of the same name wins, as setPinActivity does."""
    out = []
    pre = scope.rstrip("/") + "/"
    for var in v.vars:
        if var.type not in ("wire", "reg") or not v.values[var.id][0]:
            continue
        if not var.name.startswith(pre):
            continue
        name = var.name[len(pre):]
        if var.width == 1:
            out.append((normalize(name), var.id, 0))
            continue
        m = _BUS.match(name.replace(" ", ""))
        if not m:
            continue
        base, frm, to = m.group(1), int(m.group(2)), int(m.group(3))
        bits = range(to, frm + 1) if to < frm else range(to, frm - 1, -1)
        for vb, b in enumerate(bits):
            out.append((normalize(f"{base}[{b}]"), var.id, vb))
    return out


def normalize(name: str) -> str:
    """Escaped Verilog identifiers: drop the backslash and trailing space."""
    name = name.strip()
    parts = name.split("\\/")
    return "/".join(p[1:] if p.startswith("\\") else p for p in parts).strip()
