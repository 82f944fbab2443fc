"""Invalid events are reported through the context's status word, and the
context stays usable.

The walk checks each event it reads: times that do not increase within a
net, a time past time_max, and a window that lacks, for some net, the event
before its t_lo (its context). Each sets a bit of a device status word that
gtp_sync / gtp_fetch turn into GTP_EINVAL with a message. Every access of the
walk stays inside the net's listed range whatever the times are, so a bad
trace costs a wrong result and an error code, not a fault. After gtp_reset
the same context evaluates a valid trace exactly as the oracle does."""
import numpy as np
import pytest

from tests import toy
from tests.parity import compare

pytestmark = pytest.mark.gpu


def _case(seed=3):
    rng = np.random.default_rng(seed)
    return toy.random_design(rng, n_cell=120, n_net=50, time_max=9_000, tpc=600, wide=False)


def _read_net(d, ev):
    """A net read by some pin that lists at least four events."""
    counts = np.diff(ev.net_off)
    read = np.zeros(d.n_net if hasattr(d, "n_net") else counts.shape[0], dtype=bool)
    read[d.pin_net[d.pin_net >= 0]] = True
    nets = np.nonzero(read & (counts >= 4))[0]
    assert nets.size
    return int(nets[0])


def _events_with(ev, net, times, values):
    """A copy of ev whose net `net` lists (times, values) instead."""
    from gtpower_b200.design import Events
    vals = ev.values()
    a, b = int(ev.net_off[net]), int(ev.net_off[net + 1])
    t = np.concatenate([ev.time[:a], np.asarray(times, np.int64), ev.time[b:]])
    v = np.concatenate([vals[:a], np.asarray(values, np.uint8), vals[b:]])
    off = ev.net_off.copy()
    off[net + 1:] += len(times) - (b - a)
    return Events.from_values(off, t, v)


def _expect_einval(eng, events_list, needle):
    from gtpower_b200 import _abi
    for w in events_list:
        eng.read_power_activities(w)
    with pytest.raises(_abi.GtpError) as ex:
        eng.sync()
    assert ex.value.status == _abi.GTP_EINVAL
    assert needle in str(ex.value)


def _then_valid(eng, d, ev):
    from oracle import oracle as orc
    eng.reset()
    eng.read_power_activities(ev)
    eng.sync()
    compare(eng.fetch(counts=True), orc.run(d, ev))


def test_non_increasing_times():
    from gtpower_b200 import B200Power
    d, ev = _case()
    net = _read_net(d, ev)
    a, b = int(ev.net_off[net]), int(ev.net_off[net + 1])
    t = ev.time[a:b].copy()
    t[1], t[2] = t[2], t[1]            # one step back in time
    bad = _events_with(ev, net, t, ev.values()[a:b])
    with B200Power(d, device=0, collect_counts=True) as eng:
        _expect_einval(eng, [bad], "strictly increasing")
        _then_valid(eng, d, ev)


def test_time_past_time_max():
    from gtpower_b200 import B200Power
    d, ev = _case()
    net = _read_net(d, ev)
    a, b = int(ev.net_off[net]), int(ev.net_off[net + 1])
    t = np.concatenate([ev.time[a:b], [d.time_max + 7]])
    v = np.concatenate([ev.values()[a:b], [1 - min(1, int(ev.values()[b - 1]))]])
    bad = _events_with(ev, net, t, v)
    with B200Power(d, device=0, collect_counts=True) as eng:
        _expect_einval(eng, [bad], "beyond time_max")
        _then_valid(eng, d, ev)


def test_window_without_context():
    """The second window drops, for one net, every listed event before its
    t_lo (while saying, through net_base, that the net had earlier events)."""
    from gtpower_b200 import B200Power, windows
    from gtpower_b200.design import Events
    d, ev = _case()
    tpc = d.ticks_per_cycle
    w1, w2 = windows.split(ev, tpc, [0, 7, 16])
    t_lo = w2.t_lo
    vals = w2.values()
    # a net read by some pin whose context in w2 holds events before t_lo
    read = np.zeros(w2.net_off.shape[0] - 1, dtype=bool)
    read[d.pin_net[d.pin_net >= 0]] = True
    pick = None
    for n in np.nonzero(read)[0]:
        a, b = int(w2.net_off[n]), int(w2.net_off[n + 1])
        k = int(np.searchsorted(w2.time[a:b], t_lo))
        if k > 0 and b - a > k:
            pick = (int(n), a, b, k)
            break
    assert pick is not None
    n, a, b, k = pick
    keep = np.ones(w2.n_event, dtype=bool)
    keep[a:a + k] = False
    off = w2.net_off.copy()
    off[n + 1:] -= k
    base = w2.net_base.copy()
    base[n] += k
    bad = Events.from_values(off, w2.time[keep], vals[keep], net_base=base, t_lo=w2.t_lo, t_hi=w2.t_hi)
    with B200Power(d, device=0, collect_counts=True) as eng:
        _expect_einval(eng, [w1, bad], "lacks the event before t_lo")
        _then_valid(eng, d, ev)
