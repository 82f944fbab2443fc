"""Small hand-built designs for known-answer and edge-case tests."""
from __future__ import annotations

import numpy as np

from gtpower_b200.design import CellLibrary, Design, Events, GROUP_COMBINATIONAL, GROUP_SEQUENTIAL


def table1(axis, values):
    return {"order": 1, "axis_vars": ["slew"], "axes": [list(axis)], "values": list(values)}


def table2(ax_slew, ax_cap, values):
    return {"order": 2, "axis_vars": ["slew", "cap"], "axes": [list(ax_slew), list(ax_cap)],
            "values": list(values)}


def const(v):
    return {"order": 0, "axis_vars": [], "axes": [], "values": [v]}


def inv_cell(leak_a1=1e-9, leak_a0=2e-9, e_in_rise=None, e_in_fall=None, e_out=None,
             name="INV"):
    """Inverter A -> Y. Input energy: rise table over slew, fall constant.
    Output energy: 2-D (slew, cap) table related to A."""
    e_in_rise = e_in_rise or table1([0.0, 1e-9], [1e-15, 3e-15])
    e_in_fall = e_in_fall or const(1e-15)
    e_out = e_out or {
        "rise": table2([0.0, 1e-9], [0.0, 1e-14], [1e-14, 2e-14, 3e-14, 5e-14]),
        "fall": table2([0.0, 1e-9], [0.0, 1e-14], [2e-14, 2e-14, 4e-14, 6e-14]),
    }
    return {
        "name": name, "n_in": 1,
        "pins": [{"name": "A", "direction": "input", "capacitance": 1e-15, "clock": False},
                 {"name": "Y", "direction": "output", "capacitance": 0.0, "clock": False}],
        "internal_powers": [
            {"pin": 0, "related_pin": -1, "when": [[0, 0]], "rise": e_in_rise, "fall": e_in_fall},
            {"pin": 1, "related_pin": 0, "when": [[0, 0]], "rise": e_out["rise"], "fall": e_out["fall"]},
        ],
        "leakage_powers": [{"when": [[1, 1]], "power": leak_a1}, {"when": [[1, 0]], "power": leak_a0}],
        "cell_leakage_power": 1.5e-9, "is_sequential": False, "is_pad": False, "is_macro": False,
        "timing": [], "functions": {},
    }


def nand_cell(name="NAND2", when_tables=False):
    """NAND2 A, B -> Y with distinct tables per related pin; optionally
    `when`-conditioned input tables on A (B=1 / B=0)."""
    ip = []
    if when_tables:
        ip.append({"pin": 0, "related_pin": -1, "when": [[2, 2]], "rise": const(7e-15), "fall": const(7e-15)})
        ip.append({"pin": 0, "related_pin": -1, "when": [[2, 0]], "rise": const(5e-15), "fall": const(5e-15)})
    else:
        ip.append({"pin": 0, "related_pin": -1, "when": [[0, 0]], "rise": const(1e-15), "fall": const(2e-15)})
    ip.append({"pin": 1, "related_pin": -1, "when": [[0, 0]], "rise": const(3e-15), "fall": const(4e-15)})
    ip.append({"pin": 2, "related_pin": 0, "when": [[0, 0]], "rise": const(10e-15), "fall": const(20e-15)})
    ip.append({"pin": 2, "related_pin": 1, "when": [[0, 0]], "rise": const(30e-15), "fall": const(40e-15)})
    leaks = [{"when": [[3, s]], "power": (s + 1) * 1e-9} for s in range(4)]
    return {
        "name": name, "n_in": 2,
        "pins": [{"name": "A", "direction": "input", "capacitance": 1e-15, "clock": False},
                 {"name": "B", "direction": "input", "capacitance": 1e-15, "clock": False},
                 {"name": "Y", "direction": "output", "capacitance": 0.0, "clock": False}],
        "internal_powers": ip, "leakage_powers": leaks, "cell_leakage_power": 2.5e-9,
        "is_sequential": False, "is_pad": False, "is_macro": False, "timing": [], "functions": {},
    }


def wide_cell(n_in: int, name=None):
    """A cell with n_in inputs and one output (exercises the wide walk)."""
    pins = [{"name": f"I{k}", "direction": "input", "capacitance": 1e-15, "clock": False}
            for k in range(n_in)]
    pins.append({"name": "Z", "direction": "output", "capacitance": 0.0, "clock": False})
    ip = [{"pin": k, "related_pin": -1, "when": [[0, 0]], "rise": const((k + 1) * 1e-15),
           "fall": const((k + 2) * 1e-15)} for k in range(n_in)]
    ip += [{"pin": n_in, "related_pin": k, "when": [[0, 0]], "rise": const((k + 10) * 1e-15),
            "fall": const((k + 20) * 1e-15)} for k in range(n_in)]
    leaks = [{"when": [[1 << k, 1 << k]], "power": (k + 1) * 1e-10} for k in range(min(n_in, 4))]
    return {"name": name or f"WIDE{n_in}", "n_in": n_in, "pins": pins, "internal_powers": ip,
            "leakage_powers": leaks, "cell_leakage_power": 1e-10, "is_sequential": False,
            "is_pad": False, "is_macro": False, "timing": [], "functions": {}}


def build(cells: list[dict], instances: list[tuple[int, list[int]]], n_net: int, *,
          timescale=1e-12, period=1e-9, time_max=10_000, slew=(2e-10, 3e-10), cap=5e-15,
          volt=1.8, arcs=None, clock_pins=(), default_state=None, groups=None) -> Design:
    """instances: (type index, [net per pin]) with pins inputs-first."""
    lib = CellLibrary(cells)
    cell_type = np.asarray([t for t, _ in instances], dtype=np.int32)
    pin_off = np.zeros(len(instances) + 1, dtype=np.int32)
    pin_off[1:] = np.cumsum([len(p) for _, p in instances])
    pin_net = np.asarray([n for _, p in instances for n in p], dtype=np.int32)
    n_pin = pin_net.shape[0]
    is_out = np.zeros(n_pin, dtype=bool)
    for i, (t, _) in enumerate(instances):
        is_out[pin_off[i] + lib.n_in(t):pin_off[i + 1]] = True
    arc_off = np.zeros(len(instances), dtype=np.int64)
    arc_list = []
    for i, (t, _) in enumerate(instances):
        n_in = lib.n_in(t)
        n_out = lib.n_pin(t) - n_in
        arc_off[i] = len(arc_list)
        for o in range(n_out):
            for q in range(n_in):
                for a in range(4):
                    fr, to = a // 2, a % 2
                    if arcs is None:
                        # negative unate, 10 ps
                        arc_list.append(10e-12 if fr != to else np.nan)
                    else:
                        arc_list.append(arcs(i, o, q, fr, to))
    cp = np.zeros(n_pin, dtype=np.uint8)
    for p in clock_pins:
        cp[p] = 1
    ds = np.full(n_pin, 2, dtype=np.uint8) if default_state is None else np.asarray(default_state, np.uint8)
    return Design(
        lib=lib, timescale=timescale, clk_period=period, time_max=time_max, n_net=n_net,
        cell_type=cell_type, cell_pin_off=pin_off,
        cell_group=np.asarray(groups if groups is not None else [GROUP_COMBINATIONAL] * len(instances), np.uint8),
        cell_arc_off=arc_off, pin_net=pin_net,
        pin_slew_rise=np.full(n_pin, slew[0], np.float32), pin_slew_fall=np.full(n_pin, slew[1], np.float32),
        pin_load_cap=np.where(is_out, cap, 0.0).astype(np.float32),
        pin_voltage=np.full(n_pin, volt, np.float32), pin_default_state=ds, pin_is_clock=cp,
        arc_delay=np.asarray(arc_list if arc_list else [np.nan], dtype=np.float32))


def events(n_net: int, per_net: dict[int, list[tuple[int, int]]]) -> Events:
    off = [0]
    ts, vs = [], []
    for n in range(n_net):
        ev = per_net.get(n, [])
        for t, v in ev:
            ts.append(t)
            vs.append(v)
        off.append(len(ts))
    return Events.from_values(np.asarray(off, np.int64), np.asarray(ts, np.int64),
                              np.asarray(vs, np.uint8))


def random_design(rng: np.random.Generator, n_cell: int, n_net: int, time_max: int,
                  tpc: int, max_events: int = 40, wide: bool = True, z_values: bool = True):
    """Random small design over the toy cells with random traces (X/Z values,
    nets without events, pins without nets, same-time events)."""
    cells = [inv_cell(), nand_cell(), nand_cell("NAND2W", when_tables=True)]
    if wide:
        cells += [wide_cell(5), wide_cell(9)]
    inst = []
    for _ in range(n_cell):
        t = int(rng.integers(0, len(cells)))
        npin = len(cells[t]["pins"])
        nets = [int(rng.integers(-1, n_net)) if rng.random() < 0.05 else int(rng.integers(0, n_net))
                for _ in range(npin)]
        inst.append((t, nets))
    per = {}
    for n in range(n_net):
        if rng.random() < 0.08:
            continue  # net without events
        k = int(rng.integers(1, max_events))
        ts = np.unique(rng.integers(1, time_max + 1, size=k))
        if rng.random() < 0.85:
            ts = np.concatenate([[0], ts])
        vals = rng.choice([0, 1, 2, 3] if z_values else [0, 1, 2], size=ts.shape[0],
                          p=[0.42, 0.42, 0.1, 0.06] if z_values else [0.45, 0.45, 0.1])
        per[n] = list(zip(ts.tolist(), vals.tolist()))
    period = tpc * 1e-12
    d = build(cells, inst, n_net, period=period, time_max=time_max,
              arcs=lambda i, o, q, fr, to: (float(rng.uniform(1e-12, 4e-11))
                                           if rng.random() < 0.8 else np.nan),
              clock_pins=[p for p in range(sum(len(x[1]) for x in inst)) if rng.random() < 0.03])
    d.pin_slew_rise = rng.uniform(5e-11, 5e-10, d.n_pin).astype(np.float32)
    d.pin_slew_fall = rng.uniform(5e-11, 5e-10, d.n_pin).astype(np.float32)
    inf_mask = rng.random(d.n_pin) < 0.02
    d.pin_slew_rise[inf_mask] = np.inf
    return d, events(n_net, per)


def dff_cell(name="DFF", clk_first=False):
    """Flip-flop D, CLK -> Q (CLK first with clk_first). The clock pin's
    energies depend on D and Q (one fall energy negative), D's on the clock
    value, Q's tables are related to CLK and to D, and all 8 leakage states
    differ (the clock value included)."""
    i_d, i_c = (1, 0) if clk_first else (0, 1)
    bd, bc, bq = 1 << i_d, 1 << i_c, 1 << 2
    pins = [None, None, {"name": "Q", "direction": "output", "capacitance": 0.0, "clock": False}]
    pins[i_d] = {"name": "D", "direction": "input", "capacitance": 1e-15, "clock": False}
    pins[i_c] = {"name": "CLK", "direction": "input", "capacitance": 2e-15, "clock": True}
    ip = [
        {"pin": i_c, "related_pin": -1, "when": [[bd | bq, bd]], "rise": const(6e-15), "fall": const(2e-15)},
        {"pin": i_c, "related_pin": -1, "when": [[bd, bd]], "rise": const(5e-15), "fall": const(3e-15)},
        {"pin": i_c, "related_pin": -1, "when": [[0, 0]], "rise": table1([0.0, 1e-9], [1e-15, 4e-15]),
         "fall": const(-1e-15)},
        {"pin": i_d, "related_pin": -1, "when": [[bc, bc]], "rise": const(2e-15), "fall": const(2.5e-15)},
        {"pin": i_d, "related_pin": -1, "when": [[bc, 0]], "rise": const(1e-15), "fall": const(1.5e-15)},
        {"pin": 2, "related_pin": i_c, "when": [[0, 0]], "rise": const(20e-15), "fall": const(25e-15)},
        {"pin": 2, "related_pin": i_d, "when": [[0, 0]], "rise": const(8e-15), "fall": const(9e-15)},
    ]
    leaks = [{"when": [[7, s]], "power": (1 + s) * 1e-9 + (3e-9 if s & bc else 0.0)} for s in range(8)]
    return {"name": name, "n_in": 2, "pins": pins, "internal_powers": ip, "leakage_powers": leaks,
            "cell_leakage_power": 2e-9, "is_sequential": True, "is_pad": False, "is_macro": False,
            "timing": [], "functions": {}}


def clock_wave(tpc: int, time_max: int, pa: int, pb: int, v0: int, *, initial=True,
               gap=None) -> list[tuple[int, int]]:
    """Periodic clock: edge to 1 - v0 at phase pa and back to v0 at phase pb
    of every cycle, from an initial value at tick 0 (none: the clock is X
    until its first edge); gap = (c0, c1) drops the edges of cycles c0..c1-1
    (a stopped clock)."""
    ev = []
    if initial:
        ev.append((0, v0 if pa > 0 else 1 - v0))
    for c in range(time_max // tpc + 1):
        if gap is not None and gap[0] <= c < gap[1]:
            continue
        for ph, v in ((pa, 1 - v0), (pb, v0)):
            t = c * tpc + ph
            if 0 < t <= time_max:
                ev.append((t, v))
    return ev


def clocked_design(rng: np.random.Generator, n_dff: int, n_comb: int, n_data: int, tpc: int,
                   n_cycle: int, clocks: list[dict], tail: int = 0):
    """Random flip-flop design on periodic clocks. clocks: dicts with pa, pb,
    v0 and optional initial / gap (clock_wave). Flip-flop outputs change a
    few ticks after their clock's edges; data events fall on random ticks, a
    third of them on a clock edge; some values are X or Z. An inverter on
    each clock net (not a clock pin) reads the clock as data."""
    cells = [dff_cell(), dff_cell("DFFC", clk_first=True), inv_cell(), nand_cell()]
    time_max = n_cycle * tpc - tail
    n_clk = len(clocks)
    waves = [clock_wave(tpc, time_max, c["pa"], c["pb"], c["v0"], initial=c.get("initial", True),
                        gap=c.get("gap")) for c in clocks]
    n_q = n_dff
    d0 = n_clk                       # data nets
    q0 = n_clk + n_data              # flip-flop outputs
    x0 = q0 + n_q                    # combinational outputs
    n_net = x0 + n_comb + n_clk
    per = {k: waves[k] for k in range(n_clk)}
    edge_t = [np.asarray([t for t, _ in w if t > 0], np.int64) for w in waves]

    def data_events(k):
        n = int(rng.integers(2, 4 * n_cycle))
        ts = rng.integers(1, time_max + 1, size=n)
        snap = rng.random(n) < 0.33
        allt = np.concatenate(edge_t) if edge_t else np.zeros(0, np.int64)
        if allt.size:
            ts[snap] = rng.choice(allt, size=int(snap.sum()))
        ts = np.unique(ts)
        vals = rng.choice([0, 1, 2, 3], size=ts.size, p=[0.45, 0.45, 0.06, 0.04])
        return [(0, int(rng.integers(0, 2)))] + list(zip(ts.tolist(), vals.tolist()))

    for k in range(n_data):
        per[d0 + k] = data_events(k)
    inst = []
    for i in range(n_dff):
        ck = int(rng.integers(0, n_clk))
        d = d0 + int(rng.integers(0, n_data))
        q = q0 + i
        t = int(rng.integers(0, 2))
        inst.append((t, [ck, d, q] if t == 1 else [d, ck, q]))
        # Q follows some edges of its clock after 1..40 ticks
        et = edge_t[ck]
        qs = np.unique(np.minimum(et[rng.random(et.size) < 0.3] + int(rng.integers(1, 41)), time_max))
        per[q] = [(0, 0)] + [(int(t_), int(v)) for t_, v in zip(qs.tolist(), (np.arange(qs.size) + 1) % 2)]
    for j in range(n_comb):
        a = int(rng.integers(0, q0 + n_q))
        b = int(rng.integers(0, q0 + n_q))
        inst.append((3, [a, b, x0 + j]))
        per[x0 + j] = data_events(j)
    for k in range(n_clk):
        inst.append((2, [k, x0 + n_comb + k]))
    n_pin = sum(len(p) for _, p in inst)
    clock_pins = []
    off = 0
    for t, pins in inst:
        if t in (0, 1):
            clock_pins.append(off + (1 if t == 0 else 0))
        off += len(pins)
    d = build(cells, inst, n_net, period=tpc * 1e-12, time_max=time_max,
              arcs=lambda i, o, q, fr, to: float(rng.uniform(1e-12, 3e-11)) if rng.random() < 0.9 else np.nan,
              clock_pins=clock_pins,
              groups=[GROUP_SEQUENTIAL if t in (0, 1) else GROUP_COMBINATIONAL for t, _ in inst])
    d.pin_slew_rise = rng.uniform(5e-11, 5e-10, d.n_pin).astype(np.float32)
    d.pin_slew_fall = rng.uniform(5e-11, 5e-10, d.n_pin).astype(np.float32)
    return d, events(n_net, per)
