"""Host-side design and event containers, and their C-ABI views.

A `Design` holds what CudaPower::initGateData gathers per instance and per
pin from OpenSTA (power/cuda/CudaPower.cu:1601-1816) as numpy arrays, plus
the packed Liberty power groups of every cell type. `Events` holds the
per-net event CSR (the VcdValues each pin's PwrActivity points to,
include/sta/PowerClass.hh:44-81).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi

GROUP_COMBINATIONAL, GROUP_SEQUENTIAL, GROUP_CLOCK, GROUP_MACRO, GROUP_PAD = range(5)

_AXIS = {"slew": _abi.GTP_AXIS_SLEW, "cap": _abi.GTP_AXIS_CAP}


class CellLibrary:
    """Packs cell descriptions (liberty.Library.cell_data dicts) into the
    ABI's type / internal_power / leakage_power / table / cube pools."""

    def __init__(self, cells: list[dict]):
        self.cells = cells
        self.names = [c["name"] for c in cells]
        self.index = {n: i for i, n in enumerate(self.names)}
        lut: list[float] = []
        cubes: list[tuple[int, int]] = []
        tables = []
        types = []
        ipwrs = []
        leaks = []
        table_cache: dict[int, int] = {}

        def add_table(t) -> int:
            if t is None:
                return -1
            key = id(t)
            if key in table_cache:
                return table_cache[key]
            order = int(t["order"])
            axes = t["axes"]
            vals = t["values"]
            a1 = a2 = 0
            n1 = n2 = 1
            v1 = v2 = _abi.GTP_AXIS_NONE
            if order >= 1:
                a1 = len(lut)
                lut.extend(axes[0])
                n1 = len(axes[0])
                v1 = _AXIS.get(t["axis_vars"][0], _abi.GTP_AXIS_NONE)
            if order >= 2:
                a2 = len(lut)
                lut.extend(axes[1])
                n2 = len(axes[1])
                v2 = _AXIS.get(t["axis_vars"][1], _abi.GTP_AXIS_NONE)
            if order > 2:
                raise ValueError("3-D power tables are not supported")
            voff = len(lut)
            lut.extend(vals)
            if len(vals) != n1 * n2:
                raise ValueError("table value count does not match its axes")
            tables.append((order, v1, v2, n1, n2, a1, a2, voff))
            table_cache[key] = len(tables) - 1
            return len(tables) - 1

        def add_when(cube_list) -> tuple[int, int]:
            off = len(cubes)
            for care, val in cube_list:
                cubes.append((int(care), int(val)))
            return off, len(cube_list)

        for c in cells:
            ipwr_off = len(ipwrs)
            for ip in c["internal_powers"]:
                w = add_when(ip["when"])
                ipwrs.append((ip["pin"], ip["related_pin"], w, add_table(ip.get("rise")),
                              add_table(ip.get("fall"))))
            leak_off = len(leaks)
            for lp in c["leakage_powers"]:
                w = add_when(lp["when"])
                leaks.append((w, lp["power"]))
            clp = c.get("cell_leakage_power")
            types.append((len(c["pins"]), c["n_in"], ipwr_off, len(ipwrs) - ipwr_off, leak_off,
                          len(leaks) - leak_off, 0.0 if clp is None else clp,
                          0 if clp is None else 1))

        self.c_types = (_abi.gtp_cell_type * max(1, len(types)))()
        for i, t in enumerate(types):
            self.c_types[i] = _abi.gtp_cell_type(*t)
        self.c_ipwr = (_abi.gtp_internal_power * max(1, len(ipwrs)))()
        for i, (pin, rel, w, rt, ft) in enumerate(ipwrs):
            self.c_ipwr[i] = _abi.gtp_internal_power(pin, rel, _abi.gtp_when(*w), rt, ft)
        self.c_leak = (_abi.gtp_leakage_power * max(1, len(leaks)))()
        for i, (w, pw) in enumerate(leaks):
            self.c_leak[i] = _abi.gtp_leakage_power(_abi.gtp_when(*w), pw, 0)
        self.c_tables = (_abi.gtp_table * max(1, len(tables)))()
        for i, (o, v1, v2, n1, n2, a1, a2, vo) in enumerate(tables):
            self.c_tables[i] = _abi.gtp_table(o, v1, v2, n1, n2, a1, a2, vo, 1.0, 0)
        self.lut_pool = np.asarray(lut if lut else [0.0], dtype=np.float32)
        self.when_cubes = np.asarray(cubes if cubes else [(0, 0)], dtype=np.uint32).reshape(-1)
        self.n_type = len(types)
        self.n_ipwr = len(ipwrs)
        self.n_leak = len(leaks)
        self.n_table = len(tables)
        self.n_cube = len(cubes)

    def scaled(self, leak_scale: float = 1.0, int_scale: float = 1.0) -> "CellLibrary":
        """The same library at another corner: every internal-power table's
        scale factor times int_scale, every leakage value times leak_scale."""
        import copy
        L = copy.copy(self)
        L.c_tables = (_abi.gtp_table * len(self.c_tables))()
        for i, t in enumerate(self.c_tables):
            L.c_tables[i] = _abi.gtp_table(t.order, t.axis1_var, t.axis2_var, t.n1, t.n2, t.axis1_off,
                                           t.axis2_off, t.value_off, float(np.float32(t.scale * int_scale)), 0)
        L.c_leak = (_abi.gtp_leakage_power * len(self.c_leak))()
        for i, lp in enumerate(self.c_leak):
            L.c_leak[i] = _abi.gtp_leakage_power(lp.when, float(np.float32(lp.power * leak_scale)), 0)
        L.c_types = (_abi.gtp_cell_type * len(self.c_types))()
        for i, t in enumerate(self.c_types):
            L.c_types[i] = _abi.gtp_cell_type(t.n_pin, t.n_in, t.ipwr_off, t.n_ipwr, t.leak_off, t.n_leak,
                                              float(np.float32(t.cell_leakage_power * leak_scale)),
                                              t.has_cell_leakage_power)
        return L

    def n_pin(self, t: int) -> int:
        return len(self.cells[t]["pins"])

    def n_in(self, t: int) -> int:
        return self.cells[t]["n_in"]


@dataclass
class Design:
    lib: CellLibrary
    timescale: float                 # seconds per tick
    clk_period: float                # seconds (stored as float32)
    time_max: int
    n_net: int
    cell_type: np.ndarray            # int32 [n_cell]
    cell_pin_off: np.ndarray         # int32 [n_cell+1]
    cell_group: np.ndarray           # uint8 [n_cell]
    cell_arc_off: np.ndarray         # int64 [n_cell]
    pin_net: np.ndarray              # int32 [n_pin]
    pin_slew_rise: np.ndarray        # float32
    pin_slew_fall: np.ndarray
    pin_load_cap: np.ndarray
    pin_voltage: np.ndarray
    pin_default_state: np.ndarray    # uint8
    pin_is_clock: np.ndarray         # uint8
    arc_delay: np.ndarray            # float32
    cell_names: list[str] | None = None
    top_name: str = "top"
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_cell(self) -> int:
        return int(self.cell_type.shape[0])

    @property
    def n_pin(self) -> int:
        return int(self.pin_net.shape[0])

    @property
    def ticks_per_cycle(self) -> int:
        return int(np.ceil(np.float32(self.clk_period) / np.float32(self.timescale)))

    @property
    def n_period(self) -> int:
        return int(np.ceil((float(self.time_max) * self.timescale) / float(np.float32(self.clk_period))))

    def c_struct(self) -> _abi.gtp_design:
        """Builds the ABI struct; the arrays stay owned by this object."""
        arrs = {}

        def ptr(name, dtype):
            a = np.ascontiguousarray(getattr(self, name), dtype=dtype)
            arrs[name] = a
            return a.ctypes.data_as(C.c_void_p)

        d = _abi.gtp_design()
        d.timescale = float(self.timescale)
        d.clk_period = float(np.float32(self.clk_period))
        d.time_max = int(self.time_max)
        d.n_cell = self.n_cell
        d.n_pin = self.n_pin
        d.n_net = int(self.n_net)
        d.n_type = self.lib.n_type
        d.cell_pin_off = ptr("cell_pin_off", np.int32)
        d.cell_type = ptr("cell_type", np.int32)
        d.cell_group = ptr("cell_group", np.uint8)
        d.cell_arc_off = ptr("cell_arc_off", np.int64)
        d.pin_net = ptr("pin_net", np.int32)
        d.pin_slew_rise = ptr("pin_slew_rise", np.float32)
        d.pin_slew_fall = ptr("pin_slew_fall", np.float32)
        d.pin_load_cap = ptr("pin_load_cap", np.float32)
        d.pin_voltage = ptr("pin_voltage", np.float32)
        d.pin_default_state = ptr("pin_default_state", np.uint8)
        d.pin_is_clock = ptr("pin_is_clock", np.uint8)
        d.arc_delay = ptr("arc_delay", np.float32)
        d.n_arc_delay = int(self.arc_delay.shape[0])
        L = self.lib
        d.types = C.cast(L.c_types, C.c_void_p)
        d.internal_powers = C.cast(L.c_ipwr, C.c_void_p)
        d.leakage_powers = C.cast(L.c_leak, C.c_void_p)
        d.tables = C.cast(L.c_tables, C.c_void_p)
        d.lut_pool = L.lut_pool.ctypes.data_as(C.c_void_p)
        d.when_cubes = L.when_cubes.ctypes.data_as(C.c_void_p)
        d.n_internal_power = L.n_ipwr
        d.n_leakage_power = L.n_leak
        d.n_table = L.n_table
        d.n_when_cube = L.n_cube
        d.lut_pool_len = int(L.lut_pool.shape[0])
        self._keep = [arrs, d]
        return d


def pack_values(values: np.ndarray) -> np.ndarray:
    """One value per byte (0..3) -> 2 bits per event, 16 per uint32 word."""
    v = np.asarray(values, dtype=np.uint8)
    n = v.shape[0]
    nw = (n + 15) // 16
    pad = np.zeros(nw * 16, dtype=np.uint32)
    pad[:n] = v & 3
    pad = pad.reshape(nw, 16) << (2 * np.arange(16, dtype=np.uint32))
    return np.bitwise_or.reduce(pad, axis=1).astype(np.uint32)


def unpack_values(packed: np.ndarray, n: int) -> np.ndarray:
    w = np.asarray(packed, dtype=np.uint32)
    v = (w[:, None] >> (2 * np.arange(16, dtype=np.uint32))) & 3
    return v.reshape(-1)[:n].astype(np.uint8)


@dataclass
class Events:
    """Per-net event CSR: net n's events are time[net_off[n]:net_off[n+1]]."""
    net_off: np.ndarray      # int64 [n_net+1]
    time: np.ndarray         # int64 [n_event]
    packed: np.ndarray       # uint32 [ceil(n_event/16)]
    net_base: np.ndarray | None = None
    t_lo: int = 0
    t_hi: int = np.iinfo(np.int64).max
    _keep: list = field(default_factory=list, repr=False)

    @classmethod
    def from_values(cls, net_off, time, values, **kw) -> "Events":
        return cls(np.ascontiguousarray(net_off, dtype=np.int64),
                   np.ascontiguousarray(time, dtype=np.int64), pack_values(values), **kw)

    @property
    def n_event(self) -> int:
        return int(self.time.shape[0])

    def values(self) -> np.ndarray:
        return unpack_values(self.packed, self.n_event)

    def c_struct(self) -> _abi.gtp_events:
        e = _abi.gtp_events()
        e.n_event = self.n_event
        no = np.ascontiguousarray(self.net_off, dtype=np.int64)
        tm = np.ascontiguousarray(self.time, dtype=np.int64)
        pk = np.ascontiguousarray(self.packed, dtype=np.uint32)
        if pk.shape[0] == 0:
            pk = np.zeros(1, dtype=np.uint32)
        if tm.shape[0] == 0:
            tm = np.zeros(1, dtype=np.int64)
        e.net_off = no.ctypes.data_as(C.c_void_p)
        e.time = tm.ctypes.data_as(C.c_void_p)
        e.value_packed = pk.ctypes.data_as(C.c_void_p)
        keep = [no, tm, pk]
        if self.net_base is not None:
            nb = np.ascontiguousarray(self.net_base, dtype=np.int64)
            e.net_base = nb.ctypes.data_as(C.c_void_p)
            keep.append(nb)
        else:
            e.net_base = None
        e.t_lo = int(self.t_lo)
        e.t_hi = int(self.t_hi)
        self._keep = keep + [e]
        return e
