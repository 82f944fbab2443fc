"""The GPU trace generator produces the host stream's windows bit for bit:
same ticks, packed values, net offsets, net_base and window bounds, for
every trace mode and window size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,window,glitch", [(0, 7, 0.2), (1, 13, 0.1), (2, 50, 0.05), (3, 9, 0.3),
                                                (0, 1000, 0.05), (3, 1, 0.5)])
def test_device_windows_equal_host_stream(mode, window, glitch):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=1500, n_cycle=120, seed=4))
    spec = synth.TraceSpec(mode=mode, glitch_p=glitch, n_unit=8)
    host = synth.Stream(synth.Trace(d, info, spec, seed=7), window)
    dev = synth.DeviceStream(synth.Trace(d, info, spec, seed=7), window)
    k = 0
    while True:
        h = host.next(10_000_000)
        g = dev.next()
        if h is None:
            assert g is None
            break
        assert (g.t_lo, g.t_hi, g.n_event) == (h.t_lo, h.t_hi, h.n_event), k
        assert np.array_equal(g.net_off.cpu().numpy(), h.net_off), k
        assert np.array_equal(g.time.cpu().numpy()[:h.n_event], h.time), k
        assert np.array_equal(g.net_base.cpu().numpy(), h.net_base), k
        nw = (h.n_event + 15) // 16
        assert np.array_equal(g.packed.cpu().numpy().view(np.uint32)[:nw], h.packed[:nw]), k
        k += 1
    assert k == (120 + window - 1) // window


def test_device_windows_evaluate_like_the_whole_trace():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from gtpower_b200 import B200Power, synth
    from oracle import oracle as orc
    from tests.parity import compare
    d, info = synth.flat_design(synth.FlatSpec(n_cell=2000, n_cycle=90, seed=6))
    spec = synth.TraceSpec(mode=1, glitch_p=0.1)
    full = synth.Trace(d, info, spec, seed=3).full()
    dev = synth.DeviceStream(synth.Trace(d, info, spec, seed=3), 11)
    with B200Power(d, collect_counts=True) as eng:
        while True:
            w = dev.next()
            if w is None:
                break
            torch.cuda.synchronize()
            w.push(eng)
        eng.sync()
        res = eng.fetch(counts=True)
    compare(res, orc.run(d, full))
