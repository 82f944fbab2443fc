"""Seeded synthetic workloads for the power engine.

`flat_design` builds the levelized sky130hd netlist of the synthetic
configurations (cell mix INV 25%, NAND2 20%, NOR2 15%, AOI21 10%, XOR2 5%,
MUX2 5%, DFF 20%; fanout ~ Geometric(0.4) capped at 8; lognormal wire cap
with mean 2 fF, sigma 0.6) and annotates it with the per-pin quantities an
STA run would supply: load cap = wire cap + sum of load pin caps; each net's
slew = its driver's rise/fall_transition table at (50 ps input slew, load
cap), worst over the driver's arcs (50 ps on primary inputs and the clock);
arc delays = cell_rise / cell_fall at (input pin slew, load cap), present
for the edges the arc's timing_sense / timing_type allows.

`Trace` produces the per-net event CSR for any cycle window from a
counter-based generator, so traces of any length can be streamed.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass

import numpy as np

from . import build
from .design import CellLibrary, Design, Events, GROUP_COMBINATIONAL, GROUP_SEQUENTIAL

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "sky130hd_tt_synth_cells.json")

MIX_CELLS = [
    ("sky130_fd_sc_hd__inv_1", 0.25),
    ("sky130_fd_sc_hd__nand2_1", 0.20),
    ("sky130_fd_sc_hd__nor2_1", 0.15),
    ("sky130_fd_sc_hd__a21oi_1", 0.10),
    ("sky130_fd_sc_hd__xor2_1", 0.05),
    ("sky130_fd_sc_hd__mux2_1", 0.05),
    ("sky130_fd_sc_hd__dfxtp_1", 0.20),
]

_slib = None


def synth_lib() -> C.CDLL:
    global _slib
    if _slib is None:
        path = build.build_synth()
        L = C.CDLL(path)
        L.synth_netlist_create.restype = C.c_void_p
        L.synth_netlist_create.argtypes = [C.c_int64, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_double, C.c_int32, C.c_double,
                                           C.c_double, C.c_double]
        L.synth_netlist_size.restype = C.c_int64
        L.synth_netlist_size.argtypes = [C.c_void_p, C.c_int32]
        L.synth_netlist_copy.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        L.synth_netlist_free.argtypes = [C.c_void_p]
        L.synth_trace_create.restype = C.c_void_p
        L.synth_trace_create.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.c_int64, C.c_uint64,
                                         C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_int32, C.c_double, C.c_double, C.c_int64,
                                         C.c_int64]
        L.synth_trace_create_phased.restype = C.c_void_p
        L.synth_trace_create_phased.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.c_int64, C.c_uint64,
                                                C.c_double, C.c_double, C.c_int32, C.c_double,
                                                C.c_int32, C.c_double, C.c_double, C.c_int64, C.c_int64]
        L.synth_trace_free.argtypes = [C.c_void_p]
        L.synth_trace_phase.restype = C.c_int32
        L.synth_trace_phase.argtypes = [C.c_void_p, C.c_int64]
        L.synth_trace_count.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int32]
        L.synth_trace_fill.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_int32]
        L.synth_trace_initial.argtypes = [C.c_void_p, C.c_void_p]
        L.synth_pack_values.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int32]
        L.synth_stream_create.restype = C.c_void_p
        L.synth_stream_create.argtypes = [C.c_void_p, C.c_int64, C.c_int32]
        L.synth_stream_free.argtypes = [C.c_void_p]
        L.synth_stream_next.restype = C.c_int64
        L.synth_stream_next.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
        _slib = L
    return _slib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def load_cells(path: str = DATA) -> dict:
    with open(path) as f:
        return json.load(f)["cells"]


def _interp2(t: dict, x1: np.ndarray, x2: np.ndarray) -> np.ndarray:
    """Vectorised Table2 lookup with edge-segment extrapolation."""
    a1 = np.asarray(t["axes"][0])
    a2 = np.asarray(t["axes"][1]) if t["order"] >= 2 else np.asarray([0.0])
    v = np.asarray(t["values"]).reshape(len(a1), len(a2))
    if t["axis_vars"][0] == "cap":  # normalise to (slew, cap)
        x1, x2 = x2, x1

    def seg(a, x):
        if len(a) == 1:
            return np.zeros_like(x, dtype=np.int64), np.zeros_like(x)
        i = np.clip(np.searchsorted(a, x, side="right") - 1, 0, len(a) - 2)
        d = (x - a[i]) / (a[i + 1] - a[i])
        return i, d

    i, dx = seg(a1, x1)
    j, dy = seg(a2, x2)
    if len(a2) == 1:
        return (1 - dx) * v[i, 0] + dx * v[i + 1, 0] if len(a1) > 1 else np.full_like(x1, v[0, 0])
    return ((1 - dx) * (1 - dy) * v[i, j] + dx * (1 - dy) * v[i + 1, j]
            + dx * dy * v[i + 1, j + 1] + (1 - dx) * dy * v[i, j + 1])


def _arc_edges(timing_type: str, sense: str) -> list[tuple[int, int]]:
    """(from, to) edges of a delay arc; 0 = rise, 1 = fall."""
    if timing_type in ("rising_edge",):
        return [(0, 0), (0, 1)]
    if timing_type in ("falling_edge",):
        return [(1, 0), (1, 1)]
    if timing_type not in ("combinational", "combinational_rise", "combinational_fall",
                           "three_state_enable", "three_state_disable"):
        return []
    if sense == "positive_unate":
        return [(0, 0), (1, 1)]
    if sense == "negative_unate":
        return [(0, 1), (1, 0)]
    return [(0, 0), (0, 1), (1, 0), (1, 1)]


def annotate(lib: CellLibrary, cell_type: np.ndarray, cell_pin_off: np.ndarray,
             pin_net: np.ndarray, n_net: int, wire_cap: np.ndarray, clock_nets: set[int],
             voltage: float, input_slew: float = 50e-12):
    """Per-pin load caps, slews and per-cell arc delays from the Liberty data
    (the quantities an STA run supplies to the power walk)."""
    n_cell = cell_type.shape[0]
    n_pin = pin_net.shape[0]
    pin_cell = np.repeat(np.arange(n_cell), np.diff(cell_pin_off))
    pin_local = np.arange(n_pin) - cell_pin_off[pin_cell]
    pin_type = cell_type[pin_cell]
    cap_tab = np.zeros((lib.n_type, 64))
    is_out_tab = np.zeros((lib.n_type, 64), dtype=bool)
    clk_tab = np.zeros((lib.n_type, 64), dtype=np.uint8)
    for t, c in enumerate(lib.cells):
        for k, p in enumerate(c["pins"]):
            cap_tab[t, k] = p["capacitance"]
            is_out_tab[t, k] = k >= c["n_in"]
            clk_tab[t, k] = 1 if p["clock"] else 0
    pin_cap = cap_tab[pin_type, pin_local]
    pin_is_out = is_out_tab[pin_type, pin_local]
    pin_is_clock = clk_tab[pin_type, pin_local]
    valid = pin_net >= 0
    net_load = np.asarray(wire_cap, dtype=np.float64).copy()
    np.add.at(net_load, pin_net[valid & ~pin_is_out], pin_cap[valid & ~pin_is_out])
    load = np.where(pin_is_out & valid, net_load[np.maximum(pin_net, 0)], 0.0)

    # net slews from the driving output pin
    net_slew = np.full((2, n_net), input_slew)
    out_pins = np.nonzero(pin_is_out & valid)[0]
    for t, c in enumerate(lib.cells):
        sel = out_pins[pin_type[out_pins] == t]
        if sel.size == 0:
            continue
        for k in range(c["n_in"], len(c["pins"])):
            pk = sel[pin_local[sel] == k]
            if pk.size == 0:
                continue
            r = np.zeros(pk.size)
            f = np.zeros(pk.size)
            for tg in c["timing"]:
                if tg["pin"] != k or not _arc_edges(tg["timing_type"], tg["timing_sense"]):
                    continue
                tabs = tg["tables"]
                if "rise_transition" in tabs:
                    r = np.maximum(r, _interp2(tabs["rise_transition"], np.full(pk.size, input_slew), load[pk]))
                if "fall_transition" in tabs:
                    f = np.maximum(f, _interp2(tabs["fall_transition"], np.full(pk.size, input_slew), load[pk]))
            nets = pin_net[pk]
            net_slew[0, nets] = np.where(r > 0, r, input_slew)
            net_slew[1, nets] = np.where(f > 0, f, input_slew)
    for n in clock_nets:
        net_slew[:, n] = input_slew
    slew_r = np.where(valid, net_slew[0, np.maximum(pin_net, 0)], input_slew)
    slew_f = np.where(valid, net_slew[1, np.maximum(pin_net, 0)], input_slew)

    # arc delays [n_out][n_in][4] per cell
    n_arc = np.zeros(n_cell, dtype=np.int64)
    for t, c in enumerate(lib.cells):
        n_in = c["n_in"]
        n_out = len(c["pins"]) - n_in
        n_arc[cell_type == t] = 4 * n_in * n_out
    cell_arc_off = np.zeros(n_cell, dtype=np.int64)
    cell_arc_off[1:] = np.cumsum(n_arc)[:-1]
    arc = np.full(int(n_arc.sum()), np.nan, dtype=np.float32)
    for t, c in enumerate(lib.cells):
        cells = np.nonzero(cell_type == t)[0]
        if cells.size == 0:
            continue
        n_in = c["n_in"]
        for tg in c["timing"]:
            o = tg["pin"] - n_in
            q = tg["related_pin"]
            if o < 0 or q >= n_in:
                continue
            for fr, to in _arc_edges(tg["timing_type"], tg["timing_sense"]):
                tab = tg["tables"].get("cell_rise" if to == 0 else "cell_fall")
                if tab is None:
                    continue
                qp = cell_pin_off[cells] + q
                op = cell_pin_off[cells] + n_in + o
                s = slew_r[qp] if fr == 0 else slew_f[qp]
                dl = _interp2(tab, s, load[op])
                arc[cell_arc_off[cells] + (o * n_in + q) * 4 + 2 * fr + to] = dl.astype(np.float32)
    return (load.astype(np.float32), slew_r.astype(np.float32), slew_f.astype(np.float32),
            pin_is_clock, cell_arc_off, arc)


@dataclass
class FlatSpec:
    n_cell: int = 200_000
    n_cycle: int = 10_000
    seed: int = 20261203
    period: float = 2e-9
    timescale: float = 1e-12
    fanout_p: float = 0.4
    fanout_cap: int = 8
    wire_mean: float = 2e-15
    wire_sigma: float = 0.6
    pi_fraction: float = 0.01


def flat_design(spec: FlatSpec, cells_path: str = DATA) -> tuple[Design, dict]:
    cells = load_cells(cells_path)
    names = [n for n, _ in MIX_CELLS]
    lib = CellLibrary([cells[n] for n in names])
    mix = np.asarray([m for _, m in MIX_CELLS], dtype=np.float64)
    type_n_in = np.asarray([lib.n_in(t) for t in range(lib.n_type)], dtype=np.int32)
    type_is_ff = np.asarray([1 if cells[n]["is_sequential"] else 0 for n in names], dtype=np.int32)
    L = synth_lib()
    h = L.synth_netlist_create(spec.n_cell, spec.seed, lib.n_type, _p(mix), _p(type_n_in),
                               _p(type_is_ff), spec.fanout_p, spec.fanout_cap, spec.wire_mean,
                               spec.wire_sigma, spec.pi_fraction)
    try:
        n_cell = L.synth_netlist_size(h, 0)
        n_pin = L.synth_netlist_size(h, 1)
        n_net = L.synth_netlist_size(h, 2)
        clock_net = L.synth_netlist_size(h, 3)
        n_pi = L.synth_netlist_size(h, 4)
        cell_type = np.empty(n_cell, dtype=np.int32)
        cell_pin_off = np.empty(n_cell + 1, dtype=np.int32)
        pin_net = np.empty(n_pin, dtype=np.int32)
        wire_cap = np.empty(n_net, dtype=np.float64)
        L.synth_netlist_copy(h, _p(cell_type), _p(cell_pin_off), _p(pin_net), _p(wire_cap))
    finally:
        L.synth_netlist_free(h)
    voltage = 1.8
    load, slew_r, slew_f, pin_is_clock, cell_arc_off, arc = annotate(
        lib, cell_type, cell_pin_off, pin_net, n_net, wire_cap, {clock_net}, voltage)
    tpc = int(np.ceil(np.float32(spec.period) / np.float32(spec.timescale)))
    d = Design(
        lib=lib, timescale=spec.timescale, clk_period=float(np.float32(spec.period)),
        time_max=spec.n_cycle * tpc, n_net=n_net, cell_type=cell_type, cell_pin_off=cell_pin_off,
        cell_group=np.where(type_is_ff[cell_type] == 1, GROUP_SEQUENTIAL, GROUP_COMBINATIONAL).astype(np.uint8),
        cell_arc_off=cell_arc_off, pin_net=pin_net, pin_slew_rise=slew_r, pin_slew_fall=slew_f,
        pin_load_cap=load, pin_voltage=np.full(n_pin, voltage, dtype=np.float32),
        pin_default_state=np.full(n_pin, 2, dtype=np.uint8), pin_is_clock=pin_is_clock.astype(np.uint8),
        arc_delay=arc, top_name="synth_top")
    info = {"clock_net": int(clock_net), "n_primary_inputs": int(n_pi), "tpc": tpc,
            "n_cycle": spec.n_cycle}
    return d, info


@dataclass
class TraceSpec:
    mode: int = 0              # 0 uniform, 1 zipf+burst, 2 markov phases, 3 phased units
    lo: float = 0.05
    hi: float = 0.30
    zipf_alpha: float = 1.2
    rate_mean: float = 0.1
    burst_sigma: float = 1.5
    n_phase: int = 16
    p_stay: float = 0.99
    n_unit: int = 32           # mode 3: contiguous net ranges with per-phase activity
    act_sigma: float = 0.8     # mode 3: lognormal sigma of the activity factors
    glitch_p: float = 0.05
    w_lo_ticks: int = 5
    w_hi_ticks: int = 100


class Trace:
    """Counter-based synthetic trace over a design's nets."""

    def __init__(self, design: Design, info: dict, spec: TraceSpec, seed: int):
        self.design = design
        self.info = info
        self.spec = spec
        self.n_net = design.n_net
        self.n_cycle = info["n_cycle"]
        self.tpc = info["tpc"]
        L = synth_lib()
        if spec.mode == 3:
            self.h = L.synth_trace_create_phased(self.n_net, info["clock_net"], self.n_cycle, self.tpc,
                                                 seed, spec.lo, spec.hi, spec.n_phase, spec.p_stay,
                                                 spec.n_unit, spec.act_sigma, spec.glitch_p,
                                                 spec.w_lo_ticks, spec.w_hi_ticks)
        else:
            self.h = L.synth_trace_create(self.n_net, info["clock_net"], self.n_cycle, self.tpc, seed,
                                          spec.mode, spec.lo, spec.hi, spec.zipf_alpha, spec.rate_mean,
                                          spec.burst_sigma, spec.n_phase, spec.p_stay, spec.glitch_p,
                                          spec.w_lo_ticks, spec.w_hi_ticks)
        if not self.h:
            raise ValueError("invalid trace parameters")
        self.init = np.empty(self.n_net, dtype=np.uint8)
        L.synth_trace_initial(self.h, _p(self.init))

    def __del__(self):
        try:
            synth_lib().synth_trace_free(self.h)
        except Exception:
            pass

    def phases(self) -> np.ndarray:
        L = synth_lib()
        return np.asarray([L.synth_trace_phase(self.h, c) for c in range(self.n_cycle)], dtype=np.int32)

    def counts(self, c_lo: int, c_hi: int, threads: int = 0) -> np.ndarray:
        threads = threads or os.cpu_count() or 1
        cnt = np.empty(self.n_net, dtype=np.int64)
        synth_lib().synth_trace_count(self.h, c_lo, c_hi, _p(cnt), threads)
        return cnt

    def window(self, c_lo: int, c_hi: int, state: np.ndarray, threads: int = 0,
               out_time: np.ndarray | None = None, out_values: np.ndarray | None = None):
        """Events of cycles [c_lo, c_hi) (plus the tick-0 values when c_lo == 0).
        `state` holds each net's value before c_lo and is advanced in place."""
        threads = threads or os.cpu_count() or 1
        cnt = self.counts(c_lo, c_hi, threads)
        net_off = np.zeros(self.n_net + 1, dtype=np.int64)
        np.cumsum(cnt, out=net_off[1:])
        n = int(net_off[-1])
        times = out_time[:n] if out_time is not None else np.empty(n, dtype=np.int64)
        vals = out_values[:n] if out_values is not None else np.empty(n, dtype=np.uint8)
        synth_lib().synth_trace_fill(self.h, c_lo, c_hi, _p(net_off), _p(state), _p(times),
                                     _p(vals), threads)
        return net_off, times, vals

    def full(self, threads: int = 0) -> Events:
        state = self.init.copy()
        net_off, times, vals = self.window(0, self.n_cycle, state, threads)
        packed = np.empty((times.shape[0] + 15) // 16, dtype=np.uint32)
        synth_lib().synth_pack_values(_p(vals), times.shape[0], _p(packed), threads or os.cpu_count() or 1)
        return Events(net_off, times, packed)


class Stream:
    """Cycle windows of a `Trace` with the head/tail context each window
    needs, generated one window ahead (synth_stream_next in synth.cpp)."""

    def __init__(self, trace: Trace, window_cycles: int, threads: int = 0):
        self.trace = trace
        self.threads = threads or os.cpu_count() or 1
        self.h = synth_lib().synth_stream_create(trace.h, window_cycles, self.threads)
        self.n_net = trace.n_net

    def __del__(self):
        try:
            synth_lib().synth_stream_free(self.h)
        except Exception:
            pass

    def next_into(self, times: np.ndarray, values: np.ndarray, net_off: np.ndarray,
                  net_base: np.ndarray):
        """Fills caller buffers; returns (n_event, t_lo, t_hi), None at the
        end. Raises if the buffers are too small."""
        lo = C.c_int64()
        hi = C.c_int64()
        n = synth_lib().synth_stream_next(self.h, C.byref(lo), C.byref(hi), _p(net_off), _p(times),
                                          _p(values), _p(net_base), times.shape[0])
        if n == 0:
            return None
        if n < 0:
            raise ValueError(f"stream buffers too small: {-n} events needed")
        return int(n), lo.value, hi.value

    def next(self, cap: int) -> Events | None:
        times = np.empty(cap, np.int64)
        values = np.empty(cap, np.uint8)
        net_off = np.empty(self.n_net + 1, np.int64)
        net_base = np.empty(self.n_net, np.int64)
        r = self.next_into(times, values, net_off, net_base)
        if r is None:
            return None
        n, t_lo, t_hi = r
        packed = np.empty((n + 15) // 16, np.uint32)
        synth_lib().synth_pack_values(_p(values), n, _p(packed), self.threads)
        return Events(net_off, times[:n].copy(), packed, net_base=net_base, t_lo=t_lo, t_hi=t_hi)


# ---------------------------------------------------------------------------
# Device-side generation (synth_dev.cu): the same windows as Stream, written
# straight into device memory.

class _Rules(C.Structure):
    """ctypes mirror of gtpb::syn::Rules (csrc/synth_rules.h)."""
    _fields_ = [("mode", C.c_int32), ("clock_net", C.c_int32), ("n_net", C.c_int32), ("n_unit", C.c_int32),
                ("n_cycle", C.c_int64), ("tpc", C.c_int64), ("seed", C.c_uint64), ("lo", C.c_double),
                ("hi", C.c_double), ("glitch_p", C.c_double), ("w_lo", C.c_int64), ("w_hi", C.c_int64),
                ("net_rate", C.c_void_p), ("burst", C.c_void_p), ("phase", C.c_void_p), ("act", C.c_void_p)]


_dlib = None


def synthdev_lib() -> C.CDLL:
    global _dlib
    if _dlib is None:
        L = C.CDLL(build.build_synthdev())
        L.synthdev_create.restype = C.c_void_p
        L.synthdev_create.argtypes = [C.POINTER(_Rules), C.c_int32, C.c_int64, C.c_int32]
        L.synthdev_destroy.argtypes = [C.c_void_p]
        L.synthdev_count.restype = C.c_int64
        L.synthdev_count.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                     C.c_void_p]
        L.synthdev_fill.restype = C.c_int32
        L.synthdev_fill.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
        sl = synth_lib()
        sl.synth_trace_rules.restype = C.c_int32
        sl.synth_trace_rules.argtypes = [C.c_void_p, C.POINTER(_Rules)]
        _dlib = L
    return _dlib


@dataclass
class DeviceWindow:
    """One window of events in device memory (torch tensors), in the
    gtp_events layout: net_off int64 [n_net+1], time int64 [n_event],
    packed int32 [ceil(n_event/16)] (2-bit values), net_base int64 [n_net]."""
    c_lo: int
    c_hi: int
    t_lo: int
    t_hi: int
    n_event: int
    net_off: object
    time: object
    packed: object
    net_base: object

    def push(self, eng, t_lo: int | None = None, t_hi: int | None = None) -> None:
        """Evaluates this window (or the part [t_lo, t_hi) of it) on a
        B200Power engine."""
        eng.push_device(self.n_event, self.net_off.data_ptr(), self.time.data_ptr(), self.packed.data_ptr(),
                        self.net_base.data_ptr(), self.t_lo if t_lo is None else t_lo,
                        self.t_hi if t_hi is None else t_hi)

    def push_ranges(self, eng, ranges) -> None:
        """Evaluates only the cycle ranges [(c0, c1), ...] of this window
        (ascending, disjoint, inside it) in one pass."""
        eng.push_device_ranges(self.n_event, self.net_off.data_ptr(), self.time.data_ptr(), self.packed.data_ptr(),
                               ranges, self.net_base.data_ptr(), self.t_lo, self.t_hi)


class DeviceStream:
    """Windows of a `Trace` generated on the GPU, identical to `Stream`'s."""

    def __init__(self, trace: Trace, window_cycles: int, device: int = 0):
        import torch
        self.trace = trace
        self.device = device
        rules = _Rules()
        L = synthdev_lib()
        n_phase = synth_lib().synth_trace_rules(trace.h, C.byref(rules))
        self.h = L.synthdev_create(C.byref(rules), n_phase, window_cycles, device)
        if not self.h:
            raise RuntimeError("synthdev_create failed")
        self.n_net = trace.n_net
        self.tpc = trace.tpc
        self.n_cycle = trace.n_cycle
        self._torch = torch

    def close(self) -> None:
        if getattr(self, "h", None):
            synthdev_lib().synthdev_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def next(self, out: DeviceWindow | None = None) -> DeviceWindow | None:
        """The next window, in new tensors or, when `out` is given and large
        enough, in out's tensors (so that their addresses stay the same)."""
        torch = self._torch
        L = synthdev_lib()
        dev = f"cuda:{self.device}"
        stream = torch.cuda.current_stream(dev).cuda_stream
        net_off = out.net_off if out is not None else torch.empty(self.n_net + 1, dtype=torch.int64, device=dev)
        lo = C.c_int64()
        hi = C.c_int64()
        n = int(L.synthdev_count(self.h, net_off.data_ptr(), C.byref(lo), C.byref(hi), stream))
        if n == -1:
            return None
        if n < 0:
            raise RuntimeError("synthdev_count failed")
        if out is not None and out.time.numel() >= max(n, 1) and out.packed.numel() >= max((n + 15) // 16, 1):
            time, packed, net_base = out.time, out.packed, out.net_base
        else:
            time = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
            packed = torch.empty(max((n + 15) // 16, 1), dtype=torch.int32, device=dev)
            net_base = out.net_base if out is not None else torch.empty(self.n_net, dtype=torch.int64, device=dev)
        rc = L.synthdev_fill(self.h, net_off.data_ptr(), n, time.data_ptr(), packed.data_ptr(),
                             net_base.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"synthdev_fill failed ({rc})")
        c_lo, c_hi = lo.value, hi.value
        t_hi = c_hi * self.tpc if c_hi < self.n_cycle else np.iinfo(np.int64).max
        return DeviceWindow(c_lo, c_hi, c_lo * self.tpc, t_hi, n, net_off, time, packed, net_base)
