"""ctypes binding of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs, never by the gtpower_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.cpp")
    hdr = os.path.join(os.path.dirname(HERE), "include", "gtpb200.h")
    if force or not os.path.exists(LIB) or max(os.path.getmtime(src), os.path.getmtime(hdr)) > os.path.getmtime(LIB):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "_build/liboracle.so"], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.oracle_run.restype = C.c_int
        L.oracle_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int, C.c_int,
                                 C.c_int] + [C.c_void_p] * 11 + [C.POINTER(C.c_double)]
        L.oracle_n_period.restype = C.c_int64
        L.oracle_n_period.argtypes = [C.c_void_p]
        L.oracle_ticks_per_cycle.restype = C.c_int64
        L.oracle_ticks_per_cycle.argtypes = [C.c_void_p]
        L.oracle_table_value.restype = C.c_double
        L.oracle_table_value.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.c_float, C.c_float, C.c_int]
        L.oracle_find_value_index.restype = C.c_int64
        L.oracle_find_value_index.argtypes = [C.c_void_p, C.c_int32, C.c_float]
        L.oracle_cycle_of.restype = C.c_int64
        L.oracle_cycle_of.argtypes = [C.c_int64, C.c_double, C.c_float]
        L.oracle_n_rise.restype = C.c_float
        L.oracle_n_rise.argtypes = [C.c_int, C.c_int]
        L.oracle_n_toggle.restype = C.c_float
        L.oracle_n_toggle.argtypes = [C.c_int, C.c_int]
        L.oracle_glitch_ratio.restype = C.c_double
        L.oracle_glitch_ratio.argtypes = [C.c_int64, C.c_double, C.c_float, C.c_float, C.c_int]
        L.oracle_divergence_census.restype = C.c_int
        L.oracle_divergence_census.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        _lib = L
    return _lib


@dataclass
class OracleResult:
    cell5: np.ndarray        # [n_cell, 5] internal, glitch internal, switching, glitch switching, leakage
    cycle5: np.ndarray       # [5, n_period] leakage, internal, glitch internal, switching, glitch switching
    totals: np.ndarray       # [5] same order as cycle5
    groups: np.ndarray       # [5 groups, 5]
    cell_events: np.ndarray
    cell_glitches: np.ndarray
    cell_half_toggles: np.ndarray
    cell_related: np.ndarray
    cycle_events: np.ndarray
    cycle_glitches: np.ndarray
    dropped: int
    seconds: float


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def run(design, events, fp32: bool = False, threads: int = 1, cells: np.ndarray | None = None,
        max_leak_pins: int = 16, outputs: bool = True) -> OracleResult:
    """Runs the restated reference CPU path over `events` (one whole-trace
    window). fp32=False is the FP64 oracle; fp32=True is the reference's own
    FP32 arithmetic (the timed CPU baseline)."""
    L = lib()
    d = design.c_struct()
    e = events.c_struct()
    n_cell = design.n_cell
    npd = int(L.oracle_n_period(C.byref(d)))
    cell5 = np.zeros((n_cell, 5))
    cyc5 = np.zeros((5, max(npd, 0)))
    tot = np.zeros(5)
    grp = np.zeros((5, 5))
    ce = np.zeros(n_cell, dtype=np.uint32)
    cg = np.zeros(n_cell, dtype=np.uint32)
    ch = np.zeros(n_cell, dtype=np.uint32)
    cr = np.zeros(n_cell, dtype=np.uint32)
    ye = np.zeros(max(npd, 0), dtype=np.int64)
    yg = np.zeros(max(npd, 0), dtype=np.int64)
    dropped = np.zeros(1, dtype=np.int64)
    secs = C.c_double(0)
    sel = None
    n_sel = 0
    if cells is not None:
        sel = np.ascontiguousarray(cells, dtype=np.int32)
        n_sel = sel.shape[0]
    o = outputs
    rc = L.oracle_run(C.byref(d), C.byref(e), _p(sel) if sel is not None else None, n_sel,
                      threads, 1 if fp32 else 0, max_leak_pins,
                      _p(cell5) if o else None, _p(cyc5) if o else None, _p(tot), _p(grp),
                      _p(ce) if o else None, _p(cg) if o else None, _p(ch) if o else None,
                      _p(cr) if o else None, _p(ye) if o else None, _p(yg) if o else None,
                      _p(dropped), C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"oracle_run failed: {rc}")
    return OracleResult(cell5, cyc5, tot, grp, ce, cg, ch, cr, ye, yg, int(dropped[0]), secs.value)


CENSUS_FIELDS = ("pin_events", "toggles", "same_tick_state", "same_tick_energy",
                 "first_event_state", "glitch_class_diff", "glitch_width_diff", "related_diff",
                 "no_group_match", "beyond_cuda_cycles", "z_events")


def divergence_census(design, events, threads: int = 1) -> dict:
    """Counts the pin events on which the reference's CUDA kernel
    (power/cuda/CudaPower.cu:317-584) decides differently from its CPU path
    (power/TimeBasedPower.cc), which this package follows. Keys:
    pin_events, toggles - every walked pin event, and the toggling ones;
    same_tick_state, same_tick_energy - input toggles that the CUDA kernel
    looks up with the new values of pins toggled earlier at the same tick,
    and those among them whose energy differs; first_event_state - pins
    whose net's first event is after t=0 (the CUDA kernel takes it as the
    initial state); glitch_class_diff, glitch_width_diff - toggles that
    the CUDA per-period counters classify as glitch/non-glitch otherwise,
    or give another pulse width; related_diff - output toggles with
    another related input (delays rounded to ticks, the same-cycle rule
    for combinational cells only, near ties); no_group_match - output
    toggles with a related input and no matching `when` group (0 on the
    CPU path, the default average on CUDA); beyond_cuda_cycles - toggles
    in a cycle at or past the CUDA kernel's ceil(time_max / ticks per
    cycle) cycles, whose per-cycle terms it adds past its arrays (its last
    thread ends one tick after its last cycle); z_events - toggles to or
    from Z. The comparisons cover the events the CUDA kernel walks
    (toggles after a net's first event), with one thread over the whole
    trace."""
    L = lib()
    d = design.c_struct()
    e = events.c_struct()
    out = np.zeros(len(CENSUS_FIELDS), dtype=np.int64)
    n = L.oracle_divergence_census(C.byref(d), C.byref(e), threads, _p(out), out.shape[0])
    if n != len(CENSUS_FIELDS):
        raise RuntimeError(f"oracle_divergence_census returned {n}")
    return dict(zip(CENSUS_FIELDS, (int(v) for v in out)))


# ---- the reference's own helpers compiled from its sources (oracle/_ref) ----

REF_LIB = os.path.join(HERE, "_ref", "libref.so")
_ref = None


def build_ref(ref_root: str) -> str:
    """Compiles the reference helpers (Makefile target `ref`) from the
    reference sources under ref_root into oracle/_ref/libref.so."""
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_root}"], check=True)
    return REF_LIB


def ref_lib() -> C.CDLL | None:
    """The compiled reference helpers, or None when they were not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            return None
        L = C.CDLL(REF_LIB, mode=os.RTLD_LAZY | os.RTLD_LOCAL)
        L.ref_table1.restype = C.c_float
        L.ref_table1.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_float]
        L.ref_table2.restype = C.c_float
        L.ref_table2.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_float, C.c_float]
        L.ref_find_value_index.restype = C.c_longlong
        L.ref_find_value_index.argtypes = [C.c_void_p, C.c_int, C.c_float]
        L.ref_clked_waveform_idx.restype = C.c_longlong
        L.ref_clked_waveform_idx.argtypes = [C.c_longlong, C.c_float, C.c_float]
        L.ref_n_rise.restype = C.c_float
        L.ref_n_rise.argtypes = [C.c_int, C.c_int]
        L.ref_n_toggle.restype = C.c_float
        L.ref_n_toggle.argtypes = [C.c_int, C.c_int]
        L.ref_glitch_ratio.restype = C.c_float
        L.ref_glitch_ratio.argtypes = [C.c_float, C.c_float]
        _ref = L
    return _ref
