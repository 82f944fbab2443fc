"""Design tapes: a design, its cell library and an event CSR in one .npz.

A tape is what a GTPower run hands the power walk after STA and VCD
ingest (the per-pin arrays CudaPower::initGateData builds,
power/cuda/CudaPower.cu:1601-1816, plus the events), so a design can be
evaluated on a machine without the design's source files.
"""
from __future__ import annotations

import json

import numpy as np

from .design import CellLibrary, Design, Events

_ARRAYS = ["cell_type", "cell_pin_off", "cell_group", "cell_arc_off", "pin_net", "pin_slew_rise",
           "pin_slew_fall", "pin_load_cap", "pin_voltage", "pin_default_state", "pin_is_clock",
           "arc_delay"]


def save(path: str, design: Design, events: Events, meta: dict | None = None) -> None:
    arrs = {k: getattr(design, k) for k in _ARRAYS}
    head = {"timescale": design.timescale, "clk_period": design.clk_period,
            "time_max": int(design.time_max), "n_net": int(design.n_net),
            "top_name": design.top_name, "meta": meta or {}}
    np.savez_compressed(
        path, **arrs, ev_net_off=events.net_off, ev_time=events.time, ev_packed=events.packed,
        cells=np.frombuffer(json.dumps(design.lib.cells, separators=(",", ":")).encode(), np.uint8),
        cell_names=np.frombuffer("\n".join(design.cell_names or []).encode(), np.uint8),
        head=np.frombuffer(json.dumps(head).encode(), np.uint8))


def load(path: str) -> tuple[Design, Events, dict]:
    z = np.load(path)
    head = json.loads(z["head"].tobytes().decode())
    cells = json.loads(z["cells"].tobytes().decode())
    names = z["cell_names"].tobytes().decode()
    d = Design(lib=CellLibrary(cells), timescale=head["timescale"], clk_period=head["clk_period"],
               time_max=head["time_max"], n_net=head["n_net"],
               cell_names=names.split("\n") if names else None, top_name=head["top_name"],
               **{k: z[k] for k in _ARRAYS})
    ev = Events(z["ev_net_off"], z["ev_time"], z["ev_packed"])
    return d, ev, head["meta"]
