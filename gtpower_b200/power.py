"""Host-side mirror of GTPower's time-based Power interface over the C ABI.

    engine = B200Power(design)                 # Sta::makePower (search/Sta.cc:502-509)
    engine.read_power_activities(events)       # read_power_activities -vcd (power/Power.tcl:405-418)
    total, seq, comb, clock, macro, pad = engine.power()
                                               # Power::power (power/Power.hh:80-87)
    engine.print_cell_res(path)                # Power::printCellRes (power/Power.hh:109)
    total.print_per_cycle_results(path, top)   # PowerResult::printPerCycleResults
    print(engine.report_power())               # report_power group table (power/Power.tcl:68-90)

Every number comes from libgtpb200.so; this module only moves arrays and
formats text. Errors from the engine raise GtpError (the reference exits
the process instead).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .design import Design, Events


@dataclass
class PowerResult:
    """include/sta/PowerClass.hh:84-161. internal/switching include glitch,
    as after timeBasedPower folds them in (power/TimeBasedPower.cc:203-204)."""
    internal: float = 0.0
    glitch_internal: float = 0.0
    switching: float = 0.0
    glitch_switching: float = 0.0
    leakage: float = 0.0
    # per-cycle waveforms (W): leakage, internal, glitch internal, switching,
    # glitch switching; only on the design total
    waveforms: np.ndarray | None = None
    period: float = 0.0

    def total(self) -> float:
        return self.internal + self.switching + self.leakage

    def print_per_cycle_results(self, path: str, top_name: str, sep: str = "\t") -> None:
        """PowerResult::printPerCycleResults (include/sta/PowerClass.hh:123-149),
        written by the library (gtp_write_per_cycle_waveform)."""
        w = np.ascontiguousarray(self.waveforms if self.waveforms is not None else np.zeros((5, 0)),
                                 dtype=np.float32)
        _abi.check(_abi.lib().gtp_write_per_cycle_waveform(path.encode(), int(w.shape[1]),
                                                           w.ctypes.data_as(C.c_void_p), top_name.encode(),
                                                           sep.encode()))


def write_cell_power(path: str, design: Design, cell5: np.ndarray, sep: str = "\t") -> None:
    """cuda_cell_power.txt from per-cell results [n_cell, 5] (gtp_write_cell_power)."""
    names = design.cell_names or [f"inst{i}" for i in range(design.n_cell)]
    c_names = (C.c_char_p * max(1, len(names)))(*[n.encode() for n in names])
    t_names = (C.c_char_p * max(1, len(design.lib.names)))(*[n.encode() for n in design.lib.names])
    c5 = np.ascontiguousarray(cell5, dtype=np.float32)
    ct = np.ascontiguousarray(design.cell_type, dtype=np.int32)
    _abi.check(_abi.lib().gtp_write_cell_power(path.encode(), design.n_cell, c5.ctypes.data_as(C.c_void_p),
                                               C.cast(c_names, C.c_void_p), ct.ctypes.data_as(C.c_void_p),
                                               C.cast(t_names, C.c_void_p), sep.encode()))


@dataclass
class Counts:
    cell_events: np.ndarray
    cell_glitches: np.ndarray
    cell_half_toggles: np.ndarray
    cell_related: np.ndarray
    cycle_events: np.ndarray
    cycle_glitches: np.ndarray
    dropped: int


@dataclass
class Results:
    cell5: np.ndarray          # [n_cell, 5] Internal, Glitch_Internal, Switching, Glitch_Switching, Leakage
    cycle5: np.ndarray         # [5, n_period]
    totals: np.ndarray         # [5] FP64: leakage, internal, glitch internal, switching, glitch switching
    groups: np.ndarray         # [5 groups, 5] FP64, groups in GTP_GROUP order
    counts: Counts | None = None


class B200Power:
    """One engine context (one per host thread)."""

    def __init__(self, design: Design, *, collect_counts: bool = False, device: int = -1,
                 cycles_per_tile: int = 0, threads_per_block: int = 0, gates_per_block: int = 0,
                 max_n_pin_for_leakage_power: int = 16, sort_by_work: bool | None = None,
                 clock_runs: bool = True, split_events: int = 0, separate_kernels: bool = False,
                 warp_walk: bool = False):
        self.design = design
        L = _abi.lib()
        cfg = _abi.gtp_config()
        L.gtp_config_default(C.byref(cfg))
        cfg.cuda_device_id = device
        cfg.collect_counts = 1 if collect_counts else 0
        cfg.cycles_per_tile = cycles_per_tile
        cfg.n_thread_per_block = threads_per_block
        cfg.gates_per_block = gates_per_block
        cfg.max_n_pin_for_leakage_power = max_n_pin_for_leakage_power
        if sort_by_work is not None:
            cfg.sort_by_work = 1 if sort_by_work else 0
        # periodic clock pins walked as runs of whole cycles (False: edge by edge)
        cfg.clock_runs = 1 if clock_runs else -1
        # density split: events per thread and tile above which a cell's tile
        # is shared by several threads (0: the default 2048, -1: off)
        cfg.split_events = split_events
        # the reference's unfused evaluation (-disable_fusion): a kernel with a
        # thread per pin event for the dynamic energies, then one with a thread
        # per cell and cycle tile for the leakage
        cfg.separate_kernels = 1 if separate_kernels else 0
        # cells of up to 4 pins walked by one warp each, 32 events at a time
        # (default: one thread per cell and tile)
        cfg.warp_walk = 1 if warp_walk else 0
        self._cfg = cfg
        self._d = design.c_struct()
        ctx = C.c_void_p()
        # bound now: at interpreter exit the module globals may be gone before __del__ runs
        self._destroy = L.gtp_destroy
        _abi.check(L.gtp_create(C.byref(self._d), C.byref(cfg), C.byref(ctx)))
        self.ctx = ctx
        self.n_period = int(L.gtp_n_period(ctx))
        self.ticks_per_cycle = int(L.gtp_ticks_per_cycle(ctx))
        self._results: Results | None = None

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self._destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- activities -------------------------------------------------------
    def reset(self) -> None:
        _abi.check(_abi.lib().gtp_reset(self.ctx), self.ctx)
        self._results = None

    def read_power_activities(self, events: Events) -> None:
        """Copies one event window to the device and evaluates it."""
        e = events.c_struct()
        _abi.check(_abi.lib().gtp_push_events(self.ctx, C.byref(e)), self.ctx)
        self._results = None

    def push_device(self, n_event: int, d_net_off: int, d_time: int, d_packed: int,
                    d_net_base: int = 0, t_lo: int = 0, t_hi: int = np.iinfo(np.int64).max) -> None:
        """Evaluates a window whose arrays are already in device memory
        (raw device pointers, e.g. torch tensor .data_ptr())."""
        e = _abi.gtp_events()
        e.n_event = n_event
        e.net_off = d_net_off
        e.time = d_time
        e.value_packed = d_packed
        e.net_base = d_net_base or None
        e.t_lo = t_lo
        e.t_hi = t_hi
        _abi.check(_abi.lib().gtp_push_events_device(self.ctx, C.byref(e)), self.ctx)
        self._results = None

    def push_device_ranges(self, n_event: int, d_net_off: int, d_time: int, d_packed: int, ranges,
                           d_net_base: int = 0, t_lo: int = 0, t_hi: int = np.iinfo(np.int64).max) -> None:
        """Evaluates only the cycle ranges [(c0, c1), ...] (ascending,
        disjoint) of a device-resident window, in one pass; per-cycle power
        of other cycles stays zero."""
        r = np.ascontiguousarray(np.asarray(ranges, dtype=np.int64).reshape(-1))
        e = _abi.gtp_events()
        e.n_event = n_event
        e.net_off = d_net_off
        e.time = d_time
        e.value_packed = d_packed
        e.net_base = d_net_base or None
        e.t_lo = t_lo
        e.t_hi = t_hi
        _abi.check(_abi.lib().gtp_push_events_device_ranges(self.ctx, C.byref(e), r.ctypes.data_as(C.c_void_p),
                                                            int(r.shape[0] // 2)), self.ctx)
        self._results = None

    @property
    def stream(self) -> int:
        """cudaStream_t of the context, as an integer handle."""
        return int(_abi.lib().gtp_get_stream(self.ctx) or 0)

    def set_stream(self, stream: int | None) -> None:
        _abi.check(_abi.lib().gtp_set_stream(self.ctx, stream or None), self.ctx)

    def sync(self) -> None:
        _abi.check(_abi.lib().gtp_sync(self.ctx), self.ctx)

    # -- per-cycle waveforms by cell group ----------------------------------
    def set_cycle_groups(self, cell_group: np.ndarray | None, n_group: int = 0) -> None:
        """Keeps per-cycle waveforms per cell group as well (before the first
        window). cell_group: int32 [n_cell] in [0, n_group); None turns it off."""
        if cell_group is None:
            _abi.check(_abi.lib().gtp_set_cycle_groups(self.ctx, None, 0), self.ctx)
            return
        g = np.ascontiguousarray(cell_group, dtype=np.int32)
        assert g.shape == (self.design.n_cell,)
        _abi.check(_abi.lib().gtp_set_cycle_groups(self.ctx, g.ctypes.data_as(C.c_void_p), int(n_group)),
                   self.ctx)

    def clock_run_nets(self) -> tuple[int, int]:
        """(nets read by clock pins, those the last window walked as runs of
        whole cycles because their events were exactly periodic)."""
        n_clk, n_per = C.c_int32(0), C.c_int32(0)
        _abi.check(_abi.lib().gtp_clock_run_nets(self.ctx, C.byref(n_clk), C.byref(n_per)), self.ctx)
        return int(n_clk.value), int(n_per.value)

    def walk_items(self) -> int:
        """Threads per tile that walked the last one-window push (n_cell when
        the density split split no cell, 0 when the split is off)."""
        n = C.c_int64(0)
        _abi.check(_abi.lib().gtp_walk_items(self.ctx, C.byref(n)), self.ctx)
        return int(n.value)

    def fetch_cycle_groups(self) -> np.ndarray:
        """[n_group, 5, n_period] float32: the cycle5 rows of each group."""
        L = _abi.lib()
        ng = int(L.gtp_n_cycle_groups(self.ctx))
        out = np.zeros((ng, 5, self.n_period), dtype=np.float32)
        _abi.check(L.gtp_fetch_cycle_groups(self.ctx, out.ctypes.data_as(C.c_void_p)), self.ctx)
        return out

    # -- results ----------------------------------------------------------
    def fetch(self, counts: bool = False) -> Results:
        L = _abi.lib()
        nc = self.design.n_cell
        npd = self.n_period
        cell5 = np.zeros((nc, 5), dtype=np.float32)
        cyc5 = np.zeros((5, npd), dtype=np.float32)
        tot = np.zeros(5)
        grp = np.zeros((5, 5))
        cnt = None
        c_counts = None
        if counts:
            cnt = Counts(np.zeros(nc, np.uint32), np.zeros(nc, np.uint32), np.zeros(nc, np.uint32),
                         np.zeros(nc, np.uint32), np.zeros(npd, np.int64), np.zeros(npd, np.int64), 0)
            c_counts = _abi.gtp_counts()
            c_counts.cell_events = cnt.cell_events.ctypes.data_as(C.c_void_p)
            c_counts.cell_glitches = cnt.cell_glitches.ctypes.data_as(C.c_void_p)
            c_counts.cell_half_toggles = cnt.cell_half_toggles.ctypes.data_as(C.c_void_p)
            c_counts.cell_related = cnt.cell_related.ctypes.data_as(C.c_void_p)
            c_counts.cycle_events = cnt.cycle_events.ctypes.data_as(C.c_void_p)
            c_counts.cycle_glitches = cnt.cycle_glitches.ctypes.data_as(C.c_void_p)
        _abi.check(L.gtp_fetch(self.ctx, cell5.ctypes.data_as(C.c_void_p),
                               cyc5.ctypes.data_as(C.c_void_p), tot.ctypes.data_as(C.c_void_p),
                               grp.ctypes.data_as(C.c_void_p),
                               C.byref(c_counts) if c_counts is not None else None), self.ctx)
        if cnt is not None:
            cnt.dropped = int(c_counts.dropped)
        self._results = Results(cell5, cyc5, tot, grp, cnt)
        return self._results

    def power(self):
        """Power::power: (total, sequential, combinational, clock, macro, pad)."""
        r = self._results or self.fetch()

        def pr(v5, wave=None):
            return PowerResult(internal=float(v5[1]), glitch_internal=float(v5[2]),
                               switching=float(v5[3]), glitch_switching=float(v5[4]),
                               leakage=float(v5[0]), waveforms=wave,
                               period=float(np.float32(self.design.clk_period)))
        total = pr(r.totals, r.cycle5)
        comb, seq, clock, macro, pad = (pr(r.groups[g]) for g in range(5))
        return total, seq, comb, clock, macro, pad

    def print_cell_res(self, path: str, sep: str = "\t") -> None:
        """CudaPower::printCellRes (power/cuda/CudaPower.cu:3134-3165), written
        by the library (gtp_write_cell_power)."""
        r = self._results or self.fetch()
        write_cell_power(path, self.design, r.cell5, sep)

    def report_power(self, digits: int = 3) -> str:
        """The report_power group table (power/Power.tcl:68-90)."""
        total, seq, comb, clock, macro, pad = self.power()
        w = max(digits + 6, 10)

        def col(x):
            return f" {x:{w}.{digits}e}"

        def row(name, r):
            pct = 0.0 if total.total() == 0 else r.total() / total.total() * 100
            return (f"{name:<20s}" + col(r.internal) + col(r.switching) + col(r.leakage)
                    + col(r.total()) + f" {pct:5.1f}%")

        dashes = "-" * (20 + (w + 1) * 4)
        lines = [
            f"{'Group':<20s} {'Internal':>{w}s} {'Switching':>{w}s} {'Leakage':>{w}s} {'Total':>{w}s}",
            f"{'     ':<20s} {'Power':>{w}s} {'Power':>{w}s} {'Power':>{w}s} {'Power':>{w}s} (Watts)",
            dashes,
            row("Sequential", seq), row("Combinational", comb), row("Clock", clock),
            row("Macro", macro), row("Pad", pad), dashes, row("Total", total),
        ]

        def pcol(x):
            p = 0.0 if total.total() == 0 else x / total.total() * 100
            return f"{p:{w}.1f}%"
        lines.append(f"{'':<20s}" + pcol(total.internal) + pcol(total.switching) + pcol(total.leakage))
        return "\n".join(lines)
