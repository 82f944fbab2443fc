"""The separate dynamic and leakage kernels (gtp_config.separate_kernels, the
reference's -disable_fusion baseline: a thread per pin event for the
dynamic energies, a thread per cell and cycle tile for the leakage) against
the FP64 oracle and against the fused walk.

Counts must match the oracle bit for bit and powers within the parity
tolerance. Against the fused walk with clock pins walked edge by edge, the
per-cycle results must be bit-identical (both add the same integer
fixed-point terms) and the per-cell sums equal to FP64 rounding."""
import numpy as np
import pytest

from tests import toy
from tests.parity import close, compare

pytestmark = pytest.mark.gpu


def _oracle(d, ev):
    from oracle import oracle as orc
    return orc.run(d, ev)


def _run(d, windows, **kw):
    from gtpower_b200 import B200Power
    with B200Power(d, device=0, collect_counts=True, **kw) as eng:
        for w in windows:
            eng.read_power_activities(w)
        eng.sync()
        return eng.fetch(counts=True)


def _same_as_fused(sep, fused):
    assert np.array_equal(sep.cycle5, fused.cycle5)
    for f in ("cell_events", "cell_glitches", "cell_half_toggles", "cell_related", "cycle_events",
              "cycle_glitches"):
        assert np.array_equal(getattr(sep.counts, f), getattr(fused.counts, f)), f
    close("cell5 vs fused", sep.cell5, fused.cell5, rtol=1e-6)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_toy_designs(seed):
    """X/Z values, wide cells (8- and 32-pin buckets), pins without nets,
    nets whose first event is after tick 0, same-time events, clock pins."""
    rng = np.random.default_rng(seed)
    d, ev = toy.random_design(rng, n_cell=400, n_net=150, time_max=30_000, tpc=700)
    sep = _run(d, [ev], separate_kernels=True, cycles_per_tile=11)
    compare(sep, _oracle(d, ev))
    _same_as_fused(sep, _run(d, [ev], clock_runs=False))


def test_flat_synthetic_windows():
    """Flip-flops on a clock net, glitch pulses, the trace cut into windows
    on and off cycle boundaries; the fused walk with clock runs agrees on the
    dynamic per-cycle sums bit for bit (clock runs add the same integer
    terms) and on leakage within the fixed-point resolution."""
    from gtpower_b200 import synth, windows
    d, info = synth.flat_design(synth.FlatSpec(n_cell=3000, n_cycle=200, seed=81))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=0.1), seed=82).full()
    tpc = d.ticks_per_cycle
    cuts = [0, 41 * tpc, 97 * tpc + 501, 160 * tpc, np.iinfo(np.int64).max]
    wins = [windows.make_window(ev, tpc, cuts[k], cuts[k + 1]) for k in range(len(cuts) - 1)]
    ref = _oracle(d, ev)
    sep = _run(d, wins, separate_kernels=True)
    compare(sep, ref)
    _same_as_fused(sep, _run(d, wins, clock_runs=False))
    runs = _run(d, wins)
    assert np.array_equal(sep.cycle5[1:], runs.cycle5[1:])
    close("leakage vs clock runs", sep.cycle5[0], runs.cycle5[0], rtol=1e-6)


def test_windows_with_gaps_and_drift():
    """Windows after a gap are evaluated on their own (their leakage starts
    at their first tick); a period of 300.5 ticks drifts against the tick
    cycles. Both through the leakage kernel's walk; the fused walk must give
    the same bits."""
    from gtpower_b200 import windows
    rng = np.random.default_rng(4)
    d, ev = toy.random_design(rng, n_cell=200, n_net=60, time_max=24_000, tpc=300, wide=False)
    d.clk_period = 300.5e-12
    tpc = d.ticks_per_cycle
    spans = [(0, 20), (26, 27), (31, 55), (60, None)]
    wins = [windows.make_window(ev, tpc, c0 * tpc, c1 * tpc if c1 else np.iinfo(np.int64).max)
            for c0, c1 in spans]
    sep = _run(d, wins, separate_kernels=True)
    _same_as_fused(sep, _run(d, wins, clock_runs=False))
    # the first window continues from tick 0: its cycles equal the oracle's
    ref = _oracle(d, ev)
    close("first window", sep.cycle5[1:, :19].T, ref.cycle5[1:, :19].T)


def test_cycle_groups_and_cell_shards():
    """Per-group per-cycle waveforms, and a context restricted to a cell
    range, as with the fused walk."""
    from gtpower_b200 import B200Power, _abi
    rng = np.random.default_rng(7)
    d, ev = toy.random_design(rng, n_cell=500, n_net=120, time_max=20_000, tpc=500)
    groups = (np.arange(d.n_cell) * 7 // d.n_cell).astype(np.int32)
    out = {}
    for sep in (False, True):
        with B200Power(d, device=0, collect_counts=True, separate_kernels=sep, clock_runs=False) as eng:
            eng.set_cycle_groups(groups, 7)
            eng.read_power_activities(ev)
            eng.sync()
            out[sep] = (eng.fetch(counts=True), eng.fetch_cycle_groups())
    assert np.array_equal(out[True][1], out[False][1])
    _same_as_fused(out[True][0], out[False][0])
    with B200Power(d, device=0, collect_counts=True, separate_kernels=True) as eng:
        _abi.check(_abi.lib().gtp_set_cell_range(eng.ctx, 100, 350), eng.ctx)
        eng.read_power_activities(ev)
        eng.sync()
        part = eng.fetch(counts=True)
    assert np.all(part.counts.cell_events[:100] == 0) and np.all(part.counts.cell_events[350:] == 0)
    assert np.array_equal(part.counts.cell_events[100:350], out[True][0].counts.cell_events[100:350])
    close("shard cells", part.cell5[100:350], out[True][0].cell5[100:350], rtol=1e-6)


def test_rejected_where_only_the_fused_walk_runs():
    import torch
    from gtpower_b200 import B200Power, _abi
    rng = np.random.default_rng(3)
    d, ev = toy.random_design(rng, n_cell=50, n_net=30, time_max=5_000, tpc=500)
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(a).to(dev) for a in (ev.net_off, ev.time, ev.packed.view(np.int32))]
    with B200Power(d, device=0, separate_kernels=True) as eng:
        with pytest.raises(_abi.GtpError) as ex:
            eng.push_device_ranges(ev.n_event, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), [(1, 3)])
        assert "cycle ranges" in str(ex.value)
        # the context stays usable
        eng.read_power_activities(ev)
        eng.sync()


def test_invalid_events_reported():
    """Times that do not increase within a net: GTP_EINVAL at sync, as the
    fused walk reports it."""
    from gtpower_b200 import B200Power, _abi
    from gtpower_b200.design import Events
    rng = np.random.default_rng(2)
    d, ev = toy.random_design(rng, n_cell=60, n_net=20, time_max=5_000, tpc=500, wide=False)
    t = ev.time.copy()
    counts = np.diff(ev.net_off)
    n = next(int(x) for x in np.unique(d.pin_net[d.pin_net >= 0]) if counts[x] >= 4)
    a = int(ev.net_off[n])
    t[a + 2] = t[a + 1]
    bad = Events.from_values(ev.net_off, t, ev.values())
    with B200Power(d, device=0, separate_kernels=True) as eng:
        eng.read_power_activities(bad)
        with pytest.raises(_abi.GtpError) as exc:
            eng.sync()
        assert "strictly increasing" in str(exc.value)
