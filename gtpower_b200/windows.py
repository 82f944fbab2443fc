"""Splits a whole-trace event CSR into time windows that can be pushed one
after another (the analogue of the reference's time intervals,
power/VcdReader.cc:292-300 and power/cuda/CudaPower.cu:1263-1314).

A window covers ticks [t_lo, t_hi) on cycle boundaries. For every net it
lists, besides the events inside the window, the context the walk reads:
all events of the last clock period that has an event before t_lo plus the
event before that period (glitch grouping and related-pin edges look that
far back), and the first two events at or after t_hi (glitch look-ahead and
the end of the last leakage segment).
"""
from __future__ import annotations

import numpy as np

from .design import Events, pack_values


def window_slices(net_off: np.ndarray, time: np.ndarray, tpc: int, t_lo: int, t_hi: int):
    """Per net [ctx_start, ctx_end) indices into the whole-trace arrays."""
    n_net = net_off.shape[0] - 1
    start = np.empty(n_net, dtype=np.int64)
    end = np.empty(n_net, dtype=np.int64)
    for n in range(n_net):
        a, b = int(net_off[n]), int(net_off[n + 1])
        t = time[a:b]
        i_lo = a + int(np.searchsorted(t, t_lo, side="left"))
        i_hi = a + int(np.searchsorted(t, t_hi, side="left"))
        s = i_lo
        if i_lo > a:
            last = i_lo - 1
            p = int(time[last]) // tpc
            s = a + int(np.searchsorted(t, p * tpc, side="left"))
            s = max(a, min(s, last) - 1)
        e = min(b, i_hi + 2)
        start[n] = s
        end[n] = e
    return start, end


def make_window(events: Events, tpc: int, t_lo: int, t_hi: int) -> Events:
    vals = events.values()
    start, end = window_slices(events.net_off, events.time, tpc, t_lo, t_hi)
    counts = end - start
    off = np.zeros(counts.shape[0] + 1, dtype=np.int64)
    np.cumsum(counts, out=off[1:])
    idx = np.concatenate([np.arange(s, e) for s, e in zip(start, end)]) if off[-1] else np.zeros(0, np.int64)
    base = start - events.net_off[:-1]
    return Events(off, events.time[idx].copy(), pack_values(vals[idx]), net_base=base,
                  t_lo=t_lo, t_hi=t_hi)


def split(events: Events, tpc: int, cycle_edges: list[int]) -> list[Events]:
    """Windows at the given cycle boundaries (first 0, last past the trace)."""
    out = []
    for k in range(len(cycle_edges) - 1):
        t_lo = cycle_edges[k] * tpc
        t_hi = cycle_edges[k + 1] * tpc if k + 2 < len(cycle_edges) else np.iinfo(np.int64).max
        out.append(make_window(events, tpc, t_lo, t_hi))
    return out


def interval_edges(events: Events, tpc: int, max_events: int) -> list[int]:
    """Cycle edges [0, c1, ..., cn] of time intervals holding about
    max_events listed events each, by the reference's rule: the events are
    counted in time order, and when the count since the last cut passes
    max_events the interval ends at the time of the event that passed it,
    whose events then start nothing (power/VcdReader.cc:292-296); interval
    bounds are rounded up to cycle boundaries and empty intervals dropped
    (power/cuda/CudaPower.cu:1263-1272). The last edge is the cycle after
    the last event."""
    if max_events <= 0:
        raise ValueError("max_events must be positive")
    t = np.sort(np.asarray(events.time, dtype=np.int64))
    edges = [0]
    i = max_events                       # the (max_events + 1)-th event from the interval start
    while i < t.shape[0]:
        c = -(-int(t[i]) // tpc)         # ceil to a cycle boundary
        if c > edges[-1]:
            edges.append(c)
        i += max_events + 1
    last = (int(t[-1]) // tpc + 1) if t.shape[0] else 1
    if last > edges[-1]:
        edges.append(last)
    return edges


def split_by_events(events: Events, tpc: int, max_events: int) -> list[Events]:
    """The trace as windows with context over interval_edges(events, tpc,
    max_events); the last window runs past the trace."""
    return split(events, tpc, interval_edges(events, tpc, max_events))
