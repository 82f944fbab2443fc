"""VCD value changes read on the GPU (gtp_vcd_* in libgtpb200.so).

The header ($scope / $var declarations, timescale) is parsed on the host by
vcd.read_text; the body's value changes are tokenized, stored per id with the
reference's repeat dropping and initial value, and laid out as the engine's
per-net event CSR on the device, one list per (id, bit) source:

    raw = open(path, "rb").read()                 # gzip: decompress first
    head, body = vcd.split_header(raw)
    hdr = vcd.read_text(head.decode())
    r = GpuVcdReader(hdr, [(var_id, bit), ...])   # one source per engine net
    ev = r.parse(body)                            # device CSR
    ev.push(engine)                               # gtp_push_events_device
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from .design import Events
from .vcd import Vcd


@dataclass
class DeviceEvents:
    """The CSR of the last parse, in the reader's device memory (valid until
    its next parse or close)."""
    n_event: int
    net_off: int          # device pointers
    time: int
    packed: int
    time_max: int
    n_net: int
    _reader: object = None

    def push(self, eng) -> None:
        eng.push_device(self.n_event, self.net_off, self.time, self.packed)

    def to_host(self) -> Events:
        """A host copy (gtp_vcd_fetch), for checks."""
        off = np.zeros(self.n_net + 1, np.int64)
        t = np.zeros(max(1, self.n_event), np.int64)
        pk = np.zeros(max(1, (self.n_event + 15) // 16), np.uint32)
        _abi.check(_abi.lib().gtp_vcd_fetch(self._reader.h, off.ctypes.data_as(C.c_void_p),
                                            t.ctypes.data_as(C.c_void_p), pk.ctypes.data_as(C.c_void_p)))
        return Events(off, t[:self.n_event], pk[:(self.n_event + 15) // 16])


class GpuVcdReader:
    """The ids a VCD header declares and the (id, bit) sources wanted, as a
    device reader of VCD bodies."""

    def __init__(self, header: Vcd, sources: list[tuple[str, int]], device: int = 0):
        ids = list(dict.fromkeys(var.id for var in header.vars))
        index = {s: i for i, s in enumerate(ids)}
        enc = [s.encode() for s in ids]
        off = np.zeros(len(enc) + 1, dtype=np.int32)
        if enc:
            np.cumsum([len(b) for b in enc], out=off[1:])
        chars = b"".join(enc) or b"\0"
        src_id = np.asarray([index[vid] for vid, _ in sources], dtype=np.int32)
        src_bit = np.asarray([bit for _, bit in sources], dtype=np.int32)
        self.n_src = len(sources)
        self._keep = (chars, off, src_id, src_bit)
        self.h = None
        h = C.c_void_p()
        # bound now: at interpreter exit the module globals may be gone before __del__ runs
        self._destroy = _abi.lib().gtp_vcd_destroy
        st = _abi.lib().gtp_vcd_create(chars, off.ctypes.data_as(C.c_void_p), len(ids),
                                       src_id.ctypes.data_as(C.c_void_p), src_bit.ctypes.data_as(C.c_void_p),
                                       self.n_src, device, C.byref(h))
        if st != _abi.GTP_OK:
            raise _abi.GtpError(st, "gtp_vcd_create failed")
        self.h = h

    def parse(self, body: bytes) -> DeviceEvents:
        L = _abi.lib()
        e = _abi.gtp_events()
        tmax = C.c_int64(0)
        st = L.gtp_vcd_parse(self.h, body, len(body), C.byref(e), C.byref(tmax))
        if st != _abi.GTP_OK:
            raise _abi.GtpError(st, L.gtp_vcd_last_error(self.h).decode())
        return DeviceEvents(int(e.n_event), int(e.net_off or 0), int(e.time or 0), int(e.value_packed or 0),
                            int(tmax.value), self.n_src, self)

    def stats(self) -> tuple[int, int]:
        """(tokens, value changes before repeat dropping) of the last parse."""
        nt, nc = C.c_int64(0), C.c_int64(0)
        _abi.check(_abi.lib().gtp_vcd_stats(self.h, C.byref(nt), C.byref(nc)))
        return int(nt.value), int(nc.value)

    def close(self) -> None:
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
