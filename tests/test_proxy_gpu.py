"""Power proxy on the GPU: the tcgen05 GEMM against a torch FP32 matmul,
the training step's gradients against the CPU FP64 reference network, Adam
against its FP32 restatement, and training on a nonlinear teacher."""
import numpy as np
import pytest

from tests import mlp_ref

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    return torch


@pytest.mark.parametrize("m,n,k,bias,relu", [
    (128, 128, 64, False, False),
    (300, 200, 520, True, False),
    (1000, 512, 4096, True, True),
    (64, 40, 512, True, False),
    (257, 64, 8, False, True),
    (4096, 33, 512, True, False),
])
def test_gemm_matches_torch_fp32(m, n, k, bias, relu):
    torch = _torch()
    from gtpower_b200 import proxy
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n + k)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    bv = torch.randn(n, device="cuda", generator=g) if bias else None
    c = proxy.bf16_gemm(a, b, bv, relu)
    torch.cuda.synchronize()
    ref = a.float() @ b.float().T
    if bias:
        ref = ref + bv
    if relu:
        ref = torch.relu(ref)
    err = (c - ref).abs().max().item()
    scale = ref.abs().max().item()
    # FP32 accumulation in a different order than cuBLAS/CPU: tolerance 1e-4 of the largest entry
    assert err <= 1e-4 * scale + 1e-6, (err, scale)


def test_gemm_rejects_bad_shapes():
    torch = _torch()
    from gtpower_b200 import _abi, proxy
    a = torch.zeros(64, 12, dtype=torch.bfloat16, device="cuda")  # k = 12 is not a multiple of 8
    b = torch.zeros(64, 12, dtype=torch.bfloat16, device="cuda")
    with pytest.raises(_abi.GtpError):
        proxy.bf16_gemm(a, b)


def _teacher(rng, n, I, O):
    """Bits x ~ Bernoulli(0.3); output o is a quadratic of the count of set
    bits in a fixed subset S_o (the same subsets for every call), plus a
    linear term, so that a linear model can only fit part of it."""
    st = np.random.default_rng(99)
    subsets = [st.choice(I, 16, replace=False) for _ in range(O)]
    lin = st.normal(0, 0.05, (O, I))
    X = (rng.random((n, I)) < 0.3).astype(np.float32)
    Y = np.stack([(X[:, s].sum(1) - 4.8) ** 2 / 4.0 for s in subsets], 1) + X @ lin.T
    return X, Y.astype(np.float32)


def _proxy(I=256, H=128, O=5, B=256, **kw):
    from gtpower_b200 import proxy
    return proxy.PowerProxy(n_in=I, n_hidden=H, n_out=O, batch=B, **kw)


def test_gradients_match_fp64_reference():
    torch = _torch()
    rng = np.random.default_rng(11)
    I, H, O, B = 256, 128, 5, 256
    X, Y = _teacher(rng, 1024, I, O)
    with _proxy(I, H, O, B) as px:
        xd = torch.from_numpy(X).to("cuda", torch.bfloat16).contiguous()
        yd = torch.from_numpy(Y).cuda().contiguous()
        px.set_training_data(xd, yd)
        mean, std = px.norm()
        rows = rng.choice(1024, B, replace=False).astype(np.int32)
        loss = px.compute_grads(rows)
        g = px.unflatten(px.grads_flat())
        P = px.unflatten(px.params_flat())
        T = (Y[rows] - mean) / std
        ref_loss, ref, _ = mlp_ref.forward_backward(P.__dict__, X[rows], T.astype(np.float64), bf16=True)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        a = getattr(g, name).astype(np.float64)
        r = ref[name]
        rel = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-30)
        assert rel < 1e-2, (name, rel)
        cos = float((a * r).sum() / max(np.linalg.norm(a) * np.linalg.norm(r), 1e-30))
        assert cos > 0.9999, (name, cos)


def test_adam_step_matches_fp32_restatement():
    torch = _torch()
    rng = np.random.default_rng(12)
    I, H, O, B = 128, 64, 3, 128
    X, Y = _teacher(rng, 512, I, O)
    with _proxy(I, H, O, B, lr=2e-3) as px:
        px.set_training_data(torch.from_numpy(X).to("cuda", torch.bfloat16).contiguous(),
                             torch.from_numpy(Y).cuda().contiguous())
        p0 = px.params_flat()
        px.compute_grads(np.arange(B, dtype=np.int32))
        g = px.grads_flat()
        px.adam_step()
        p1 = px.params_flat()
    ref, _, _ = mlp_ref.adam_update(p0, g, np.zeros_like(p0), np.zeros_like(p0), 1, 2e-3, 0.9, 0.999, 1e-8)
    assert np.allclose(p1, ref, rtol=1e-5, atol=1e-7)


def test_training_beats_linear_fit_on_nonlinear_teacher():
    torch = _torch()
    rng = np.random.default_rng(13)
    I, H, O, B = 256, 128, 5, 256
    X, Y = _teacher(rng, 8192, I, O)
    Xte, Yte = _teacher(np.random.default_rng(14), 2048, I, O)
    with _proxy(I, H, O, B, lr=2e-3) as px:
        px.set_training_data(torch.from_numpy(X).to("cuda", torch.bfloat16).contiguous(),
                             torch.from_numpy(Y).cuda().contiguous())
        losses = px.train(40)
        pred = px.predict(torch.from_numpy(Xte).to("cuda", torch.bfloat16).contiguous()).cpu().numpy()
    assert losses[-1] < 0.25 * losses[0], losses
    # least-squares linear model on the same features
    Xa = np.hstack([X, np.ones((len(X), 1), np.float32)]).astype(np.float64)
    W, *_ = np.linalg.lstsq(Xa, Y.astype(np.float64), rcond=None)
    lin = np.hstack([Xte, np.ones((len(Xte), 1), np.float32)]) @ W
    rmse_mlp = np.sqrt(np.mean((pred - Yte) ** 2))
    rmse_lin = np.sqrt(np.mean((lin - Yte) ** 2))
    assert rmse_mlp < 0.8 * rmse_lin, (rmse_mlp, rmse_lin)


def test_graph_and_eager_training_agree():
    torch = _torch()
    rng = np.random.default_rng(15)
    I, H, O, B = 128, 64, 3, 128
    X, Y = _teacher(rng, 1024, I, O)
    xd = torch.from_numpy(X).to("cuda", torch.bfloat16).contiguous()
    yd = torch.from_numpy(Y).cuda().contiguous()
    out = []
    for g in (True, False):
        with _proxy(I, H, O, B, use_graph=g) as px:
            px.set_training_data(xd, yd)
            px.train(3)
            out.append(px.params_flat())
    assert np.allclose(out[0], out[1], rtol=1e-5, atol=1e-6)


def test_toggle_bits_and_stats_from_event_csr():
    torch = _torch()
    from gtpower_b200 import proxy
    tpc = 100
    # net 0: initial + toggles in cycles 1, 1, 3; net 1: initial only; net 2: cycle 0 and 4
    off = np.array([0, 4, 5, 8], np.int64)
    t = np.array([0, 150, 160, 310, 0, 0, 20, 499], np.int64)
    d_off = torch.from_numpy(off).cuda()
    d_t = torch.from_numpy(t).cuda()
    sel = torch.tensor([2, 0, 1], dtype=torch.int32, device="cuda")
    x = proxy.toggle_bits(d_off, d_t, sel, tpc, 0, 5).float().cpu().numpy()
    want = np.zeros((5, 3), np.float32)
    want[[0, 4], 0] = 1
    want[[1, 3], 1] = 1
    assert np.array_equal(x, want)
    y = torch.tensor([1.0, 2.0, 4.0, 8.0, 16.0], device="cuda")
    cnt, s = proxy.net_toggle_stats(d_off, d_t, 3, tpc, 0, 5, y)
    assert cnt.cpu().tolist() == [2, 0, 2]
    assert s.cpu().tolist() == [2.0 + 8.0, 0.0, 1.0 + 16.0]
    # windowed: cycles [2, 5) only
    x2 = proxy.toggle_bits(d_off, d_t, sel, tpc, 2, 5).float().cpu().numpy()
    assert np.array_equal(x2, want[2:5])


@pytest.mark.parametrize("n_sel", [64, 70, 130, 520])
def test_dense_toggle_bits_of_windows_match_per_window_bits(n_sel):
    """gtp_toggle_bits_windows against gtp_toggle_bits window by window: an
    odd net count (a partial last group of 256, an odd row stride), a window
    longer than one 2048-row chunk, events outside the windows, rows outside
    every window left as they were."""
    torch = _torch()
    from gtpower_b200 import proxy
    rng = np.random.default_rng(21 + n_sel)
    tpc, n_net, n_cyc = 50, 600, 6000
    sel = torch.from_numpy(rng.choice(n_net, n_sel, replace=False).astype(np.int32)).cuda()
    windows, ref = [], torch.zeros((n_cyc, n_sel), dtype=torch.bfloat16, device="cuda")
    cuts = [100, 900, 3700, 3701, 5500]           # rows [0, 100) and [5500, 6000) belong to no window
    for lo, hi in zip(cuts[:-1], cuts[1:]):
        counts = rng.integers(0, 60, n_net)
        off = np.zeros(n_net + 1, np.int64)
        off[1:] = np.cumsum(counts)
        t = np.concatenate([np.sort(rng.choice(np.arange((lo - 3) * tpc, (hi + 3) * tpc), c, replace=False))
                            for c in counts]).astype(np.int64)
        d_off, d_t = torch.from_numpy(off).cuda(), torch.from_numpy(t).cuda()
        windows.append((d_off, d_t, lo, hi))
        proxy.toggle_bits(d_off, d_t, sel, tpc, lo, hi, out=ref[lo:])
    out = torch.full((n_cyc, n_sel), 7.0, dtype=torch.bfloat16, device="cuda")
    proxy.toggle_bits_windows(windows, sel, tpc, 0, out)
    torch.cuda.synchronize()
    assert torch.equal(out[100:5500], ref[100:5500])
    assert bool((out[:100] == 7.0).all()) and bool((out[5500:] == 7.0).all())
    assert float(ref.float().sum()) > 0


@pytest.mark.parametrize("I,H,O,n", [(256, 192, 5, 1000), (128, 64, 3, 333), (512, 512, 33, 4100)])
def test_predict_matches_bf16_fp64_reference(I, H, O, n):
    """Inference through the BF16 hidden layers (written by TMA stores of
    staged 32 x 64 boxes): row counts that end inside a tile, hidden widths
    below, at and above one column tile, against the FP64 network with the
    same BF16 roundings."""
    torch = _torch()
    rng = np.random.default_rng(I + H + n)
    X, Y = _teacher(rng, n, I, O)
    with _proxy(I, H, O, 256) as px:
        xd = torch.from_numpy(X).to("cuda", torch.bfloat16).contiguous()
        px.set_training_data(xd, torch.from_numpy(Y).cuda().contiguous())
        mean, std = px.norm()
        got = px.predict(xd).cpu().numpy().astype(np.float64)
        P = px.unflatten(px.params_flat())
    _, _, Ys = mlp_ref.forward_backward(P.__dict__, X.astype(np.float64), np.zeros((n, O)), bf16=True)
    ref = Ys * std.astype(np.float64) + mean.astype(np.float64)
    scale = np.abs(ref).max()
    err = np.abs(got - ref).max()
    # FP32 vs FP64 accumulation, then BF16 roundings of the hidden layers that
    # may land on either side: 1e-2 of the largest output
    assert err <= 1e-2 * scale, (err, scale)
    # and no row or column out of place: the error is small everywhere
    assert np.median(np.abs(got - ref)) <= 1e-3 * scale
