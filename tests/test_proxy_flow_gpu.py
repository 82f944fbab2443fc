"""The learned proxy end to end on a phased-unit workload (100k cells): engine
labels, correlation selection, training on the tcgen05 kernels, inference,
audit. Checks what the network gains over the linear model on the same
selected toggle bits, and that the engine's spot evaluation of audit ranges
reproduces the full-trace labels."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_proxy_flow_phased_workload():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from gtpower_b200 import proxy_flow as pf
    from gtpower_b200 import synth
    d, info = synth.flat_design(synth.FlatSpec(n_cell=100000, n_cycle=12000, seed=31))
    spec = synth.TraceSpec(mode=3, lo=0.02, hi=0.12, n_phase=16, p_stay=0.99, n_unit=16, act_sigma=1.0)
    tr = synth.Trace(d, info, spec, seed=32)
    wins = pf.generate_on_device(tr, 1000)
    assert sum(w.c_hi - w.c_lo for w in wins) == 12000
    rep = pf.run_flow(d, wins, info["tpc"], n_train=9000, n_block=16, k=2048, hidden=256, batch=512,
                      epochs=40, lr=1e-3, audit_frac=0.02, audit_run=10, seed=3,
                      exclude=(info["clock_net"],))
    print(rep)
    # the engine evaluated on the spot ranges equals the full-trace labels
    assert rep.spot_max_rel < 1e-5
    assert rep.losses[-1] < rep.losses[0]
    # the network beats the linear model on the same inputs
    assert rep.nrmse_total < rep.linear_nrmse_total
    assert rep.nrmse_blocks < rep.linear_nrmse_blocks
    assert rep.nrmse_total < 0.02
    assert rep.total_power_error < 0.005
