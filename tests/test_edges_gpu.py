"""Edge cases of the walk against the FP64 oracle: a design without cells,
one and two ticks per cycle (the division fast paths), an empty window
between windows, events at time_max on a cycle boundary, one very dense net
over many tiles, the widest cell the walk takes (32 pins) and the first one
it rejects."""
import numpy as np
import pytest

from tests import toy
from tests.parity import compare

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


def _random_events(rng, n_net, time_max, k_max, start_at_zero=True):
    per = {}
    for n in range(n_net):
        k = int(rng.integers(1, k_max))
        ts = np.unique(rng.integers(1, time_max + 1, size=k))
        if start_at_zero:
            ts = np.concatenate([[0], ts])
        vals = rng.choice([0, 1, 2], size=ts.shape[0], p=[0.45, 0.45, 0.1])
        per[n] = list(zip(ts.tolist(), vals.tolist()))
    return per


def test_design_without_cells():
    d = toy.build([toy.inv_cell()], [], 3, time_max=5_000)
    ev = toy.events(3, {0: [(0, 0), (100, 1)], 2: [(0, 1), (4_000, 0)]})
    res = _run(d, [ev])
    assert res.cell5.size == 0
    assert np.all(res.cycle5 == 0) and np.all(res.totals == 0)


@pytest.mark.parametrize("tpc", [1, 2, 3])
def test_few_ticks_per_cycle(tpc):
    rng = np.random.default_rng(tpc)
    cells = [toy.inv_cell(), toy.nand_cell()]
    n_net = 40
    inst = [(int(t), [int(x) for x in rng.integers(0, n_net, 2 + int(t))]) for t in rng.integers(0, 2, 120)]
    time_max = 900
    d = toy.build(cells, inst, n_net, period=tpc * 1e-12, time_max=time_max)
    assert d.ticks_per_cycle == tpc
    ev = toy.events(n_net, _random_events(rng, n_net, time_max, 60))
    compare(_run(d, [ev]), _oracle(d, ev))
    compare(_run(d, [ev], cycles_per_tile=7), _oracle(d, ev))


def test_empty_window_between_windows():
    from gtpower_b200 import windows
    rng = np.random.default_rng(4)
    cells = [toy.inv_cell(), toy.nand_cell()]
    n_net = 30
    inst = [(int(t), [int(x) for x in rng.integers(0, n_net, 2 + int(t))]) for t in rng.integers(0, 2, 80)]
    tpc, time_max = 500, 20_000
    d = toy.build(cells, inst, n_net, period=tpc * 1e-12, time_max=time_max)
    per = {}
    for n in range(n_net):
        early = np.unique(rng.integers(1, 6_000, 12))
        late = np.unique(rng.integers(14_000, time_max + 1, 12))
        ts = np.concatenate([[0], early, late])
        per[n] = list(zip(ts.tolist(), rng.integers(0, 2, ts.shape[0]).tolist()))
    ev = toy.events(n_net, per)
    cuts = [0, 6_500, 13_500, np.iinfo(np.int64).max]      # [6500, 13500) holds no event
    wins = [windows.make_window(ev, tpc, cuts[k], cuts[k + 1]) for k in range(3)]
    assert wins[1].n_event == 0 or np.all((wins[1].time < 6_500) | (wins[1].time >= 13_500))
    compare(_run(d, wins), _oracle(d, ev))


def test_events_at_time_max_on_a_cycle_boundary():
    rng = np.random.default_rng(6)
    cells = [toy.inv_cell(), toy.nand_cell()]
    n_net = 20
    inst = [(int(t), [int(x) for x in rng.integers(0, n_net, 2 + int(t))]) for t in rng.integers(0, 2, 60)]
    tpc = 400
    time_max = 25 * tpc
    d = toy.build(cells, inst, n_net, period=tpc * 1e-12, time_max=time_max)
    per = _random_events(rng, n_net, time_max - 1, 30)
    for n in range(0, n_net, 3):    # a third of the nets change at time_max
        v = 1 - per[n][-1][1] if per[n][-1][1] < 2 else 0
        per[n].append((time_max, v))
    ev = toy.events(n_net, per)
    compare(_run(d, [ev]), _oracle(d, ev))


def test_one_dense_net_over_many_tiles():
    """One inverter on a net with 200k events (a toggle every 3 ticks on
    average, several per cycle: glitch groups everywhere)."""
    rng = np.random.default_rng(8)
    time_max = 600_000
    ts = np.unique(rng.integers(1, time_max + 1, 200_000))
    vals = np.arange(ts.shape[0]) % 2
    per = {0: [(0, 0)] + list(zip(ts.tolist(), vals.tolist())), 1: [(0, 1), (time_max, 0)]}
    d = toy.build([toy.inv_cell(), toy.nand_cell()], [(0, [0, 1]), (1, [0, 1, 2])], 3,
                  period=1e-9, time_max=time_max)
    ev = toy.events(3, per)
    compare(_run(d, [ev]), _oracle(d, ev))
    compare(_run(d, [ev], cycles_per_tile=17), _oracle(d, ev))


def test_widest_cell_and_the_first_rejected():
    from gtpower_b200 import B200Power, _abi
    rng = np.random.default_rng(10)
    n_net = 40
    cells = [toy.wide_cell(31), toy.inv_cell()]      # 32 pins: the widest walked
    inst = [(0, [int(x) for x in rng.integers(0, n_net, 32)]) for _ in range(20)]
    inst += [(1, [int(x) for x in rng.integers(0, n_net, 2)]) for _ in range(20)]
    d = toy.build(cells, inst, n_net, period=700e-12, time_max=30_000)
    ev = toy.events(n_net, _random_events(rng, n_net, 30_000, 50))
    compare(_run(d, [ev]), _oracle(d, ev))
    d33 = toy.build([toy.wide_cell(32)], [(0, list(range(33)))], 33, time_max=1_000)
    with pytest.raises(_abi.GtpError):
        B200Power(d33, device=0)
