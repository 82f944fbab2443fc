"""The GPU VCD reader against the host reader (gtpower_b200/vcd.py, the
reference's value semantics) on random VCD text: for every (id, bit)
source the event list, times and 2-bit values, must be the same, and so
must time_max; the CSR then drives the engine like the host-built one.
Plus the header split on the host (no GPU)."""
import numpy as np
import pytest

from tests import vcd_gen


def _host_lists(text, sources):
    from gtpower_b200 import vcd
    v = vcd.read_text(text)
    return v, [vcd.bit_values(v, vid, bit) for vid, bit in sources]


def test_split_header_then_read_text_equals_read(tmp_path):
    from gtpower_b200 import vcd
    rng = np.random.default_rng(1)
    text, sources = vcd_gen.make_vcd(rng, n_steps=40)
    p = tmp_path / "a.vcd"
    p.write_text(text)
    whole = vcd.read(str(p))
    head, body = vcd.split_header(text.encode())
    assert head + body == text.encode()
    assert head.rstrip().endswith(b"$end") and b"$enddefinitions" in head
    hv = vcd.read_text(head.decode())
    assert [x.id for x in hv.vars] == [x.id for x in whole.vars]
    assert hv.timescale == whole.timescale
    assert body.lstrip().startswith(b"#0")


def test_bus_values_saturate_as_strtol_reads_them():
    from gtpower_b200 import vcd
    text = ("$timescale 1ps $end\n$var wire 70 ! v [69:0] $end\n$enddefinitions $end\n"
            "#0\nb" + "1" * 70 + " !\n#3\nb1 !\n")
    v = vcd.read_text(text)
    assert v.values["!"][2][:2] == [(1 << 63) - 1, 1]


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_gpu_reader_equals_host_reader(seed):
    from gtpower_b200 import vcd
    from gtpower_b200.vcd_gpu import GpuVcdReader
    rng = np.random.default_rng(seed)
    text, sources = vcd_gen.make_vcd(rng, n_scalar=25 + 10 * seed, n_vec=8, n_steps=150 * seed)
    hv, lists = _host_lists(text, sources)
    head, body = vcd.split_header(text.encode())
    with GpuVcdReader(vcd.read_text(head.decode()), sources, device=0) as r:
        dev = r.parse(body)
        got = dev.to_host()
        n_tok, n_ch = r.stats()
    assert dev.time_max == hv.time_max
    assert n_tok == len(body.split())
    vals = got.values()
    for s, (t_ref, v_ref) in enumerate(lists):
        a, b = int(got.net_off[s]), int(got.net_off[s + 1])
        assert np.array_equal(got.time[a:b], t_ref), s
        assert np.array_equal(vals[a:b], v_ref), s
    assert dev.n_event == sum(t.shape[0] for t, _ in lists)


@pytest.mark.gpu
def test_gpu_reader_feeds_the_engine():
    """Cells reading the parsed nets: the engine on the GPU-built CSR gives
    the same results as on the host reader's CSR."""
    from gtpower_b200 import B200Power, vcd
    from gtpower_b200.design import Events
    from gtpower_b200.vcd_gpu import GpuVcdReader
    from tests import toy
    rng = np.random.default_rng(9)
    text, sources = vcd_gen.make_vcd(rng, n_scalar=60, n_vec=0, n_real=0, n_steps=300, p_change=0.2)
    hv, lists = _host_lists(text, sources)
    # same-time double changes give non-increasing times: drop those sources
    keep = [s for s, (t, _) in enumerate(lists) if np.all(np.diff(t) > 0)]
    sources = [sources[s] for s in keep]
    lists = [lists[s] for s in keep]
    n_net = len(sources)
    off = np.concatenate([[0], np.cumsum([t.shape[0] for t, _ in lists])]).astype(np.int64)
    host_ev = Events.from_values(off, np.concatenate([t for t, _ in lists]), np.concatenate([v for _, v in lists]))
    tmax = int(max(hv.time_max, int(host_ev.time.max())))
    cells = [toy.inv_cell(), toy.nand_cell()]
    inst = []
    for _ in range(200):
        t = int(rng.integers(0, 2))
        inst.append((t, [int(x) for x in rng.integers(0, n_net, len(cells[t]["pins"]))]))
    d = toy.build(cells, inst, n_net, period=200e-12, time_max=tmax)
    head, body = vcd.split_header(text.encode())
    with GpuVcdReader(vcd.read_text(head.decode()), sources, device=0) as r:
        dev = r.parse(body)
        with B200Power(d, device=0, collect_counts=True) as eng:
            dev.push(eng)
            eng.sync()
            got = eng.fetch(counts=True)
    with B200Power(d, device=0, collect_counts=True) as eng:
        eng.read_power_activities(host_ev)
        eng.sync()
        ref = eng.fetch(counts=True)
    assert np.array_equal(got.cycle5, ref.cycle5)
    assert np.array_equal(got.cell5, ref.cell5)
    assert np.array_equal(got.counts.cell_events, ref.counts.cell_events)


@pytest.mark.gpu
def test_gpu_reader_rejects_undeclared_id():
    from gtpower_b200 import _abi, vcd
    from gtpower_b200.vcd_gpu import GpuVcdReader
    text = "$timescale 1ns $end\n$var wire 1 ! a $end\n$enddefinitions $end\n#0\n1!\n#5\n0?\n"
    head, body = vcd.split_header(text.encode())
    with GpuVcdReader(vcd.read_text(head.decode()), [("!", 0)], device=0) as r:
        with pytest.raises(_abi.GtpError) as ex:
            r.parse(body)
        assert "undeclared id" in str(ex.value)
        ok = r.parse(b"#0\n1!\n#7\n0!\n")      # the reader stays usable
        assert ok.n_event == 2 and ok.time_max == 7
