"""Many designs' traces evaluated together on one GPU.

- BatchPower: one window per engine per push, walked in one persistent
  launch per pin bucket from a device work queue (gtp_batch_*), with the
  launch sequence replayed from a CUDA graph while the window buffers stay.
- fold_corner: library corners that scale the internal-power tables and the
  leakage values. Internal and leakage energies are linear in those values
  (table interpolation, the default average over tables and the state-time
  weighting of leakage are all linear; which table applies does not depend
  on its values), so one walk gives every such corner: internal and glitch
  internal scale with the internal factor, leakage with the leakage factor,
  switching (C V^2) is unchanged.
- tune: the autotuner. It times candidate tile and block shapes on a sample
  of the batch's first windows and returns the fastest.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _abi
from .power import B200Power, Results

# corner (leakage scale, internal-power scale)
CORNERS = ((0.8, 0.8), (1.0, 1.0), (1.3, 1.3))


def _bind():
    L = _abi.lib()
    if getattr(L, "_batch_bound", False):
        return L
    P = C.c_void_p
    sigs = {
        "gtp_batch_config_default": ([C.POINTER(_abi.gtp_batch_config)], None),
        "gtp_batch_create": ([C.POINTER(C.c_void_p), C.c_int32, C.POINTER(_abi.gtp_batch_config),
                              C.POINTER(C.c_void_p)], C.c_int32),
        "gtp_batch_destroy": ([P], None),
        "gtp_batch_last_error": ([P], C.c_char_p),
        "gtp_batch_push_device": ([P, P], C.c_int32),
        "gtp_batch_sync": ([P], C.c_int32),
        "gtp_batch_get_stream": ([P], P),
        "gtp_batch_stats": ([P, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int32),
    }
    for name, (a, r) in sigs.items():
        f = getattr(L, name)
        f.argtypes = a
        f.restype = r
    L._batch_bound = True
    return L


def fold_corner(res: Results, leak_scale: float, int_scale: float) -> Results:
    """Results of the corner whose leakage values are scaled by leak_scale
    and internal-power tables by int_scale."""
    cell5 = res.cell5.astype(np.float64).copy()
    cell5[:, 0:2] *= int_scale      # Internal, Glitch_Internal
    cell5[:, 4] *= leak_scale       # Leakage
    cyc = res.cycle5.astype(np.float64).copy()
    cyc[0] *= leak_scale            # leakage
    cyc[1:3] *= int_scale           # internal, glitch internal
    tot = res.totals.copy()
    tot[0] *= leak_scale
    tot[1:3] *= int_scale
    grp = res.groups.copy()
    grp[:, 0] *= leak_scale
    grp[:, 1:3] *= int_scale
    return Results(cell5.astype(np.float32), cyc.astype(np.float32), tot, grp, res.counts)


class BatchPower:
    """A batch over engines (B200Power) that share a device and block shape."""

    def __init__(self, engines: list[B200Power], use_graph: bool = True, blocks_per_sm: int = 0):
        L = _bind()
        self.engines = engines
        cfg = _abi.gtp_batch_config()
        L.gtp_batch_config_default(C.byref(cfg))
        cfg.use_graph = 1 if use_graph else 0
        cfg.blocks_per_sm = blocks_per_sm
        arr = (C.c_void_p * len(engines))(*[e.ctx.value for e in engines])
        h = C.c_void_p()
        st = L.gtp_batch_create(arr, len(engines), C.byref(cfg), C.byref(h))
        if st != _abi.GTP_OK:
            raise _abi.GtpError(st, (L.gtp_last_error(None) or b"").decode())
        self.h = h
        self._ev = (_abi.gtp_events * len(engines))()

    def close(self) -> None:
        if getattr(self, "h", None):
            _bind().gtp_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != _abi.GTP_OK:
            msg = _bind().gtp_batch_last_error(self.h)
            raise _abi.GtpError(st, msg.decode() if msg else "")

    @property
    def stream(self) -> int:
        return int(_bind().gtp_batch_get_stream(self.h) or 0)

    def push(self, windows) -> None:
        """windows[i]: a synth.DeviceWindow for engine i, or None to skip it."""
        for i, w in enumerate(windows):
            e = self._ev[i]
            if w is None:
                e.net_off = None
                e.n_event = 0
                continue
            e.n_event = w.n_event
            e.net_off = w.net_off.data_ptr()
            e.time = w.time.data_ptr()
            e.value_packed = w.packed.data_ptr()
            e.net_base = w.net_base.data_ptr()
            e.t_lo = w.t_lo
            e.t_hi = w.t_hi
        self._check(_bind().gtp_batch_push_device(self.h, self._ev))
        for e in self.engines:
            e._results = None

    def sync(self) -> None:
        self._check(_bind().gtp_batch_sync(self.h))

    def stats(self) -> dict:
        items = C.c_int64()
        launches = C.c_int32()
        replays = C.c_int32()
        self._check(_bind().gtp_batch_stats(self.h, C.byref(items), C.byref(launches), C.byref(replays)))
        return {"items": items.value, "launches": launches.value, "graph_replays": replays.value}


@dataclass
class Shape:
    cycles_per_tile: int
    threads_per_block: int
    gates_per_block: int

    def engine_kw(self) -> dict:
        return dict(cycles_per_tile=self.cycles_per_tile, threads_per_block=self.threads_per_block,
                    gates_per_block=self.gates_per_block)


DEFAULT_CANDIDATES = (Shape(512, 256, 256), Shape(768, 256, 256), Shape(512, 256, 1024), Shape(256, 256, 256),
                      Shape(1024, 256, 256), Shape(512, 128, 256))


def tune(designs, windows, candidates=DEFAULT_CANDIDATES, repeats: int = 2, log=None):
    """Times each candidate shape on the given first windows (one per
    design, device memory) through a batch and returns (best Shape, table of
    (shape, seconds)). Each trial resets its engines, so the windows can be
    pushed again."""
    import torch
    say = log or (lambda *a: None)
    table = []
    for cand in candidates:
        engines = [B200Power(d, **cand.engine_kw()) for d in designs]
        try:
            with BatchPower(engines) as bp:
                s = torch.cuda.ExternalStream(bp.stream)
                best = float("inf")
                for r in range(repeats + 1):
                    for e in engines:
                        e.reset()
                    torch.cuda.synchronize()
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(s)
                    bp.push(windows)
                    b.record(s)
                    bp.sync()
                    if r > 0:  # the first push captures the graph
                        best = min(best, a.elapsed_time(b) / 1e3)
        finally:
            for e in engines:
                e.close()
        table.append((cand, best))
        say(f"tune {cand}: {best * 1e3:.2f} ms")
    best = min(table, key=lambda x: x[1])[0]
    return best, table


def run_sequential(engines, windows) -> float:
    """The same windows pushed engine by engine (one launch sequence per
    design); device seconds on a common stream, for comparison."""
    import torch
    s = torch.cuda.Stream()
    for e in engines:
        e.set_stream(s.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for e, w in zip(engines, windows):
        if w is not None:
            w.push(e)
    b.record(s)
    s.synchronize()
    for e in engines:
        e.set_stream(None)
    return a.elapsed_time(b) / 1e3
