"""C-ABI library: loads, exports every declared symbol, validates designs
before touching the device (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from gtpower_b200 import _abi
from tests import toy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    inc = os.path.join(ROOT, "include")
    hdr = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(gtp_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    L = _abi.lib()
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(_abi.EXPORTED) == syms


def test_struct_layout_matches_c_compiler(tmp_path):
    # the ctypes mirror must agree with the C compiler's layout of the header
    import subprocess
    names = ["gtp_table", "gtp_when", "gtp_internal_power", "gtp_leakage_power",
             "gtp_cell_type", "gtp_design", "gtp_events", "gtp_config", "gtp_counts",
             "gtp_proxy_config", "gtp_batch_config"]
    src = tmp_path / "sz.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gtpb200.h"',
             '#include "gtpb200_proxy.h"', "int main(void){"]
    for n in names:
        lines.append(f'printf("{n} %zu\\n", sizeof({n}));')
    for f, _ in _abi.gtp_design._fields_:
        lines.append(f'printf("gtp_design.{f} %zu\\n", offsetof(gtp_design, {f}));')
    for f, _ in _abi.gtp_config._fields_:
        lines.append(f'printf("gtp_config.{f} %zu\\n", offsetof(gtp_config, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for n in names:
        assert C.sizeof(getattr(_abi, n)) == int(out[n]), n
    for f, _ in _abi.gtp_design._fields_:
        assert getattr(_abi.gtp_design, f).offset == int(out[f"gtp_design.{f}"]), f
    for f, _ in _abi.gtp_config._fields_:
        assert getattr(_abi.gtp_config, f).offset == int(out[f"gtp_config.{f}"]), f


def _create(design, **cfg_fields):
    L = _abi.lib()
    d = design.c_struct()
    cfg = _abi.gtp_config()
    L.gtp_config_default(C.byref(cfg))
    for k, v in cfg_fields.items():
        setattr(cfg, k, v)
    ctx = C.c_void_p()
    st = L.gtp_create(C.byref(d), C.byref(cfg), C.byref(ctx))
    if st == 0:
        L.gtp_destroy(ctx)
    return st, L.gtp_last_error(None).decode()


def small():
    return toy.build([toy.inv_cell(), toy.nand_cell()], [(0, [0, 1]), (1, [0, 1, 2])], 3)


def test_rejects_bad_pin_count():
    d = small()
    d.cell_pin_off = np.asarray([0, 2, 4], np.int32)  # NAND2 needs 3 pins
    d.pin_net = d.pin_net[:4]
    d.pin_slew_rise = d.pin_slew_rise[:4]
    d.pin_slew_fall = d.pin_slew_fall[:4]
    d.pin_load_cap = d.pin_load_cap[:4]
    d.pin_voltage = d.pin_voltage[:4]
    d.pin_default_state = d.pin_default_state[:4]
    d.pin_is_clock = d.pin_is_clock[:4]
    st, msg = _create(d)
    assert st == _abi.GTP_EINVAL and "pin count" in msg


def test_rejects_net_out_of_range():
    d = small()
    d.pin_net = d.pin_net.copy()
    d.pin_net[0] = 99
    st, msg = _create(d)
    assert st == _abi.GTP_EINVAL and "net" in msg


def test_rejects_bad_time_base():
    d = small()
    d.time_max = 0
    st, msg = _create(d)
    assert st == _abi.GTP_EINVAL


def test_rejects_bad_type():
    d = small()
    d.cell_type = np.asarray([0, 7], np.int32)
    st, msg = _create(d)
    assert st == _abi.GTP_EINVAL and "type" in msg


def test_rejects_bad_default_state():
    d = small()
    d.pin_default_state = d.pin_default_state.copy()
    d.pin_default_state[1] = 3
    st, msg = _create(d)
    assert st == _abi.GTP_EINVAL


@pytest.mark.parametrize("threads", [512, 1024, 48, 16, -32])
def test_rejects_block_size_the_walk_cannot_launch(threads):
    # the walk kernels are compiled for blocks of at most 256 threads, in
    # warps; the check comes before any device work
    st, msg = _create(small(), n_thread_per_block=threads)
    assert st == _abi.GTP_EINVAL and "n_thread_per_block" in msg


def test_pack_values_roundtrip():
    from gtpower_b200.design import pack_values, unpack_values
    rng = np.random.default_rng(0)
    for n in (0, 1, 15, 16, 17, 1000):
        v = rng.integers(0, 4, n).astype(np.uint8)
        p = pack_values(v)
        assert np.array_equal(unpack_values(p, n), v)
        out = np.zeros(max(1, (n + 15) // 16), np.uint32)
        _abi.lib().gtp_pack_values(v.ctypes.data_as(C.c_void_p), n, out.ctypes.data_as(C.c_void_p))
        assert np.array_equal(out[:p.shape[0]], p)
