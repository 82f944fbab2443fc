"""One design's cells sharded across GPUs, one process per GPU.

Cells are independent given their pins' event lists (the reference walks
them in any order over a thread pool, power/Power.cc:262-340), so rank r of
N walks a contiguous cell range and the ranks add their accumulators once:

    shards = partition_cells(design, N, net_counts)      # same on every rank
    eng = ShardedPower(design, rank, N, pg)               # B200Power + cell range
    eng.read_power_activities(shard_events(design, ev, *shards[rank]))
    res = eng.fetch()                                     # the whole design's results

The accumulator block of each rank (gtp_export_accumulators) is summed with
one collective per element type: FP64 all-reduce of the per-cell sums (each
cell is non-zero on one rank only, so the sum is exact) and 64-bit integer
all-reduces of the fixed-point per-cycle bins and of the counters (exact and
order-independent). Every rank then imports the sum and finalizes the same
results. With NCCL over NVLink the exchange is (40 B x cells + 48 B x
cycles), about 8.5 MB for 200k cells x 10k cycles. A rank receives the
events of the nets its cells read; nets read by several shards are
replicated, read-only.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .design import Design, Events, pack_values
from .power import B200Power


def _cell_pin_events(design: Design, net_counts: np.ndarray | None) -> np.ndarray:
    """Work estimate per cell: its pins' events (or its pin count without counts)."""
    off = design.cell_pin_off
    if net_counts is None:
        return np.diff(off).astype(np.int64)
    p = design.pin_net
    pe = np.where(p >= 0, np.asarray(net_counts, np.int64)[np.maximum(p, 0)], 0)
    return np.add.reduceat(pe, off[:-1]) if design.n_cell else np.zeros(0, np.int64)


def partition_cells(design: Design, n_shard: int, net_counts: np.ndarray | None = None) -> list[tuple[int, int]]:
    """Contiguous cell ranges [begin, end), one per shard, of about equal work
    (pin events when per-net event counts are given, else pins)."""
    if n_shard < 1:
        raise ValueError("n_shard must be >= 1")
    w = _cell_pin_events(design, net_counts).astype(np.float64) + 1.0
    cum = np.concatenate([[0.0], np.cumsum(w)])
    cuts = [0]
    for r in range(1, n_shard):
        cuts.append(int(np.searchsorted(cum, cum[-1] * r / n_shard, side="left")))
    cuts.append(design.n_cell)
    cuts = np.maximum.accumulate(np.clip(np.asarray(cuts), 0, design.n_cell))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(n_shard)]


def shard_nets(design: Design, begin: int, end: int) -> np.ndarray:
    """Boolean mask of the nets that cells [begin, end) read."""
    m = np.zeros(design.n_net, dtype=bool)
    p = design.pin_net[design.cell_pin_off[begin]:design.cell_pin_off[end]]
    m[p[p >= 0]] = True
    return m


def shard_events(design: Design, events: Events, begin: int, end: int) -> Events:
    """The window `events` with only the nets that cells [begin, end) read
    (the other nets list no events); net ids are unchanged."""
    keep = shard_nets(design, begin, end)
    cnt = np.diff(events.net_off)
    cnt_new = np.where(keep, cnt, 0)
    off = np.zeros_like(events.net_off)
    np.cumsum(cnt_new, out=off[1:])
    sel = np.repeat(keep, cnt)
    vals = events.values()[sel]
    return Events(off, events.time[sel].copy(), pack_values(vals),
                  net_base=None if events.net_base is None else events.net_base.copy(),
                  t_lo=events.t_lo, t_hi=events.t_hi)


def accumulator_segments(n_cell: int, n_period: int, counts: bool) -> list[tuple[str, int, int, str]]:
    """(name, byte offset, element count, dtype) of the accumulator block,
    in the layout gtp_export_accumulators writes."""
    segs = [("cell", 5 * n_cell, "float64"), ("cycle", 6 * (n_period + 1), "int64")]
    if counts:
        segs += [("cycle_counts", 2 * (n_period + 1), "int64"), ("cell_counts", 4 * n_cell, "int32")]
    out, off = [], 0
    for name, n, dt in segs:
        out.append((name, off, n, dt))
        off += n * np.dtype(dt).itemsize
    return out


def all_reduce_block(block, segments, pg) -> None:
    """Sums a flat uint8 torch tensor laid out as `segments` over the ranks of
    process group `pg` (torch.distributed), one collective per segment: FP64
    for the per-cell sums, int64 for the fixed-point bins and the counters
    (uint64 counters add the same in two's complement), int32 for the
    per-cell counters."""
    import torch
    for name, off, n, dt in segments:
        if n == 0:
            continue
        nb = n * np.dtype(dt).itemsize
        view = block[off:off + nb].view({"float64": torch.float64, "int64": torch.int64,
                                         "int32": torch.int32}[dt])
        pg.all_reduce(view, op=pg.ReduceOp.SUM)


class ShardedPower:
    """The engine on one rank of a cell-sharded design: a B200Power over the
    whole design restricted to cells [begin, end)."""

    def __init__(self, design: Design, rank: int, world: int, pg=None, shards=None, **engine_kw):
        import torch
        self.design = design
        self.rank, self.world, self.pg = rank, world, pg
        self.shards = shards or partition_cells(design, world)
        self.begin, self.end = self.shards[rank]
        self.engine = B200Power(design, **engine_kw)
        L = _abi.lib()
        _abi.check(L.gtp_set_cell_range(self.engine.ctx, self.begin, self.end), self.engine.ctx)
        self.n_bytes = int(L.gtp_accumulator_bytes(self.engine.ctx))
        dev = engine_kw.get("device", -1)
        self.device = torch.device("cuda", dev if dev >= 0 else torch.cuda.current_device())
        self.segments = accumulator_segments(design.n_cell, self.engine.n_period,
                                             bool(engine_kw.get("collect_counts", False)))
        self._reduced = False

    def read_power_activities(self, events: Events) -> None:
        self.engine.read_power_activities(events)
        self._reduced = False

    def push_device(self, *a, **kw) -> None:
        self.engine.push_device(*a, **kw)
        self._reduced = False

    def reset(self) -> None:
        self.engine.reset()
        self._reduced = False

    def export_block(self):
        """This rank's accumulators as a flat uint8 device tensor."""
        import torch
        blk = torch.empty(self.n_bytes, dtype=torch.uint8, device=self.device)
        _abi.check(_abi.lib().gtp_export_accumulators(self.engine.ctx, C.c_void_p(blk.data_ptr())),
                   self.engine.ctx)
        self.engine.sync()
        return blk

    def import_block(self, blk) -> None:
        _abi.check(_abi.lib().gtp_import_accumulators(self.engine.ctx, C.c_void_p(blk.data_ptr())),
                   self.engine.ctx)

    def reduce(self) -> None:
        """Sums the accumulators over the ranks (one collective per element
        type) and imports the sum, so that fetch() returns the whole design."""
        import torch
        blk = self.export_block()
        if self.pg is not None and self.world > 1:
            all_reduce_block(blk, self.segments, self.pg)
            # the collectives ran on torch's stream: done before the import
            torch.cuda.current_stream(self.device).synchronize()
        self.import_block(blk)

    def fetch(self, counts: bool = False):
        """The whole design's results (every rank takes the same collective
        steps: call it on all ranks)."""
        if not self._reduced:
            self.reduce()
            self._reduced = True
        return self.engine.fetch(counts=counts)

    def close(self) -> None:
        self.engine.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
