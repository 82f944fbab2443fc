"""GPU parity: the CUDA engine against the FP64 oracle on the same inputs."""
import numpy as np
import pytest

from tests import toy
from tests.parity import compare

pytestmark = pytest.mark.gpu


def run_engine(design, windows, **kw):
    from gtpower_b200 import B200Power
    with B200Power(design, collect_counts=True, **kw) as eng:
        for w in windows:
            eng.read_power_activities(w)
        eng.sync()
        return eng.fetch(counts=True)


def oracle(design, events):
    from oracle import oracle as orc
    return orc.run(design, events)


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
@pytest.mark.parametrize("cycles_per_tile", [0, 3, 17])
def test_random_toy_designs(seed, cycles_per_tile):
    rng = np.random.default_rng(seed)
    d, ev = toy.random_design(rng, n_cell=300, n_net=120, time_max=20_000, tpc=700)
    res = run_engine(d, [ev], cycles_per_tile=cycles_per_tile)
    compare(res, oracle(d, ev))


@pytest.mark.parametrize("seed", [5, 6])
def test_random_toy_windows(seed):
    from gtpower_b200 import windows
    rng = np.random.default_rng(seed)
    d, ev = toy.random_design(rng, n_cell=200, n_net=90, time_max=15_000, tpc=500)
    tpc = d.ticks_per_cycle
    wins = windows.split(ev, tpc, [0, 3, 11, 12, 20, 31])
    res = run_engine(d, wins, cycles_per_tile=4)
    compare(res, oracle(d, ev))


@pytest.mark.parametrize("n_cell,n_cycle", [(500, 60), (3000, 120)])
def test_synthetic_flat(n_cell, n_cycle):
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=n_cell, n_cycle=n_cycle, seed=n_cell))
    ev = synth.Trace(d, info, synth.TraceSpec(), seed=n_cycle).full()
    res = run_engine(d, [ev])
    compare(res, oracle(d, ev))


def test_synthetic_skew_windows():
    from gtpower_b200 import synth, windows
    d, info = synth.flat_design(synth.FlatSpec(n_cell=1500, n_cycle=80, seed=3))
    ev = synth.Trace(d, info, synth.TraceSpec(mode=1, glitch_p=0.1), seed=9).full()
    wins = windows.split(ev, d.ticks_per_cycle, [0, 17, 40, 41, 80])
    res = run_engine(d, wins, cycles_per_tile=8)
    compare(res, oracle(d, ev))


def test_empty_trace():
    d = toy.build([toy.inv_cell()], [(0, [0, 1]), (0, [-1, 2])], 3)
    ev = toy.events(3, {})
    res = run_engine(d, [ev])
    compare(res, oracle(d, ev))


@pytest.mark.parametrize("window", [9, 25])
def test_streamed_skew_trace(window):
    """Skewed (Zipf x burst) trace pushed window by window from the streaming
    generator equals the oracle on the whole trace."""
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=2000, n_cycle=100, seed=8))
    spec = synth.TraceSpec(mode=1, glitch_p=0.1)
    full = synth.Trace(d, info, spec, seed=12).full()
    st = synth.Stream(synth.Trace(d, info, spec, seed=12), window)
    wins = []
    while True:
        w = st.next(400_000)
        if w is None:
            break
        wins.append(w)
    res = run_engine(d, wins, cycles_per_tile=6)
    compare(res, oracle(d, full))


@pytest.mark.parametrize("sort_by_work", [True, False])
@pytest.mark.parametrize("n_group,layout,gpb", [(4, "blocks", 0), (7, "blocks", 64), (5, "random", 0),
                                                (500, "random", 0)])
def test_cycle_groups_match_oracle_on_cell_subsets(n_group, layout, gpb, sort_by_work):
    """Per-cycle waveforms by cell group equal the oracle restricted to each
    group's cells; the whole-design waveforms are unchanged. 500 groups over
    3000 cells make every block span many groups (the global-memory path)."""
    from gtpower_b200 import B200Power, synth, windows
    from oracle import oracle as orc
    from tests.parity import close
    d, info = synth.flat_design(synth.FlatSpec(n_cell=3000, n_cycle=90, seed=21))
    ev = synth.Trace(d, info, synth.TraceSpec(glitch_p=0.1), seed=22).full()
    if layout == "blocks":
        grp = (np.arange(d.n_cell) * n_group // d.n_cell).astype(np.int32)
    else:
        grp = np.random.default_rng(n_group).integers(0, n_group, d.n_cell).astype(np.int32)
    wins = windows.split(ev, d.ticks_per_cycle, [0, 31, 90])
    with B200Power(d, gates_per_block=gpb, cycles_per_tile=16, sort_by_work=sort_by_work) as eng:
        eng.set_cycle_groups(grp, n_group)
        for w in wins:
            eng.read_power_activities(w)
        res = eng.fetch()
        G = eng.fetch_cycle_groups()
    full = orc.run(d, ev)
    close("cycle5", res.cycle5.T, full.cycle5.T)
    close("totals", res.totals, full.totals)
    # Per-event energies are FP32 (the reference's float table values), so a
    # group sum that nearly cancels (negative fall energies) carries FP32
    # rounding relative to its terms: values below 1e-3 of the whole
    # design's column maximum are held to 1e-8 of that maximum.
    scale = np.max(np.abs(full.cycle5.T), axis=0, keepdims=True)
    for g in sorted(set(grp.tolist()))[:12]:
        o = orc.run(d, ev, cells=np.nonzero(grp == g)[0])
        ref = o.cycle5.T
        tol = 1e-5 * np.maximum(np.abs(ref), 1e-3 * scale)
        err = np.abs(G[g].T.astype(np.float64) - ref)
        assert (err <= tol).all(), (g, np.argwhere(err > tol)[:5].tolist())
    close("sum of groups", G.sum(0).T, full.cycle5.T)


def test_host_buffers_may_be_reused_when_push_returns():
    """gtp_push_events reads caller memory only until it returns (its copies
    overlap the previous window's walk): scribbling over each window's host
    arrays right after the push leaves the results unchanged."""
    import torch
    from gtpower_b200 import B200Power, synth
    from gtpower_b200.design import Events
    d, info = synth.flat_design(synth.FlatSpec(n_cell=2500, n_cycle=120, seed=17))
    spec = synth.TraceSpec(mode=1, glitch_p=0.1)
    full = synth.Trace(d, info, spec, seed=18).full()
    st = synth.Stream(synth.Trace(d, info, spec, seed=18), 13)
    with B200Power(d, collect_counts=True, cycles_per_tile=5) as eng:
        while True:
            w = st.next(2_000_000)
            if w is None:
                break
            pin = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
                   for a in (w.net_off, w.time, w.packed.view(np.int32), w.net_base)]
            ev = Events(pin[0].numpy(), pin[1].numpy(), pin[2].numpy().view(np.uint32), net_base=pin[3].numpy(),
                        t_lo=w.t_lo, t_hi=w.t_hi)
            eng.read_power_activities(ev)
            for p in pin[1:]:
                p.fill_(-1)
        eng.sync()
        res = eng.fetch(counts=True)
    compare(res, oracle(d, full))
