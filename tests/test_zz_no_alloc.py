"""gtp_evaluate_noalloc: the allocation-free entry point.

Callers that cannot allocate device memory while they run (an EDA host
whose device memory is one arena reserved at start-up, or a service that
cannot absorb the device-wide synchronization cudaMalloc/cudaFree may
cause) evaluate a trace through gtp_evaluate_noalloc, which keeps its
accumulators in a static device array and writes into buffers the caller
owns. This test calls it through the C ABI twice in a row (the second call
must not see the first call's accumulators) and checks both against the
regular entry points within the parity tolerance. The file name sorts last
so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_path_twice():
    import torch
    from gtpower_b200 import B200Power, _abi, synth
    from tests.parity import close

    d, info = synth.flat_design(synth.FlatSpec(n_cell=3000, n_cycle=150, seed=21))
    ev = synth.Trace(d, info, synth.TraceSpec(), seed=22).full()
    with B200Power(d, device=0) as eng:
        eng.read_power_activities(ev)
        ref = eng.fetch()

        dev = torch.device("cuda", 0)
        d_off = torch.from_numpy(ev.net_off).to(dev)
        d_t = torch.from_numpy(ev.time).to(dev)
        d_v = torch.from_numpy(ev.packed.view(np.int32)).to(dev)
        npd = eng.n_period
        e = _abi.gtp_events()
        e.n_event = ev.n_event
        e.net_off = d_off.data_ptr()
        e.time = d_t.data_ptr()
        e.value_packed = d_v.data_ptr()
        e.net_base = None
        e.t_lo = 0
        e.t_hi = np.iinfo(np.int64).max
        L = _abi.lib()
        free_before = None
        for call in range(2):
            cell5 = torch.full((d.n_cell, 5), float("nan"), dtype=torch.float32, device=dev)
            cyc5 = torch.full((5, npd), float("nan"), dtype=torch.float32, device=dev)
            tot = torch.zeros(5, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            if call == 1:
                free_before = torch.cuda.mem_get_info(0)[0]
            st = L.gtp_evaluate_noalloc(eng.ctx, C.byref(e), cell5.data_ptr(), cyc5.data_ptr(),
                                        tot.data_ptr())
            _abi.check(st, eng.ctx)
            eng.sync()
            if call == 1:
                # no device memory was taken by the call
                assert torch.cuda.mem_get_info(0)[0] == free_before
            close(f"cell5 call {call}", cell5.cpu().numpy(), ref.cell5, rtol=1e-6)
            close(f"cycle5 call {call}", cyc5.cpu().numpy().T, ref.cycle5.T, rtol=1e-6)
            close(f"totals call {call}", tot.cpu().numpy(), ref.totals, rtol=1e-9)


def test_noalloc_rejects_design_beyond_scratch():
    from gtpower_b200 import B200Power, _abi, synth

    d, info = synth.flat_design(synth.FlatSpec(n_cell=500_000, n_cycle=4, seed=3))
    with B200Power(d, device=0) as eng:
        e = _abi.gtp_events()
        e.n_event = 0
        e.net_off = 1          # never dereferenced: the size check comes first
        e.t_lo = 0
        e.t_hi = 10
        st = _abi.lib().gtp_evaluate_noalloc(eng.ctx, C.byref(e), None, None, None)
        assert st == _abi.GTP_EOVERFLOW
        assert "scratch" in _abi.lib().gtp_last_error(eng.ctx).decode()


def test_noalloc_reports_invalid_events_then_runs_clean():
    """A trace whose times step back within a net makes gtp_sync report
    GTP_EINVAL after the allocation-free call; the next call with a valid
    trace starts from a clear status word and matches the regular path."""
    import torch
    from gtpower_b200 import B200Power, _abi, synth
    from tests.parity import close

    d, info = synth.flat_design(synth.FlatSpec(n_cell=2000, n_cycle=80, seed=31))
    ev = synth.Trace(d, info, synth.TraceSpec(), seed=32).full()
    read = np.zeros(d.n_net, dtype=bool)
    read[d.pin_net[d.pin_net >= 0]] = True
    counts = np.diff(ev.net_off)
    net = int(np.nonzero(read & (counts >= 4) & (np.arange(d.n_net) != info["clock_net"]))[0][0])
    a = int(ev.net_off[net])
    bad_t = ev.time.copy()
    bad_t[a + 1], bad_t[a + 2] = bad_t[a + 2], bad_t[a + 1]
    dev = torch.device("cuda", 0)
    with B200Power(d, device=0) as eng:
        eng.read_power_activities(ev)
        ref = eng.fetch()
        L = _abi.lib()
        npd = eng.n_period
        cell5 = torch.zeros((d.n_cell, 5), dtype=torch.float32, device=dev)
        cyc5 = torch.zeros((5, npd), dtype=torch.float32, device=dev)
        d_off = torch.from_numpy(ev.net_off).to(dev)
        d_v = torch.from_numpy(ev.packed.view(np.int32)).to(dev)
        for times, ok in ((bad_t, False), (ev.time, True)):
            d_t = torch.from_numpy(np.ascontiguousarray(times)).to(dev)
            e = _abi.gtp_events()
            e.n_event = ev.n_event
            e.net_off = d_off.data_ptr()
            e.time = d_t.data_ptr()
            e.value_packed = d_v.data_ptr()
            e.net_base = None
            e.t_lo = 0
            e.t_hi = np.iinfo(np.int64).max
            _abi.check(L.gtp_evaluate_noalloc(eng.ctx, C.byref(e), cell5.data_ptr(), cyc5.data_ptr(), None),
                       eng.ctx)
            if not ok:
                with pytest.raises(_abi.GtpError) as ex:
                    eng.sync()
                assert ex.value.status == _abi.GTP_EINVAL
                assert "strictly increasing" in str(ex.value)
            else:
                eng.sync()
                close("cell5", cell5.cpu().numpy(), ref.cell5, rtol=1e-6)
                close("cycle5", cyc5.cpu().numpy().T, ref.cycle5.T, rtol=1e-6)
