"""Learned per-cycle power proxy, end to end on one GPU.

1. The trace is streamed window by window (synth.Stream) into device-resident
   event CSRs (DeviceWindow).
2. The engine (the plain time-based power walk) labels the training cycles
   with per-cycle total power and the power of n_block contiguous cell
   blocks (gtp_set_cycle_groups).
3. Nets are selected by the correlation of their per-cycle toggle bit with
   each label (gtp_net_toggle_stats), a quota per output, then by the
   correlation with the total.
4. Per-cycle toggle bits of the selected nets (gtp_toggle_bits) are the
   network's inputs; the BF16 MLP (gtp_proxy_*) trains on the labelled
   cycles and predicts the rest.
5. The engine stays the authority: cycles whose input activity lies outside the
   training range and an audit sample are recomputed with it.

Every step runs in libgtpb200.so kernels; torch tensors hold device memory and
numpy holds small host-side summaries.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import proxy as px
from . import synth
from .power import B200Power
from .synth import DeviceWindow


def _torch():
    import torch
    return torch


def generate_on_device(trace: synth.Trace, window_cycles: int, device: int = 0) -> list[DeviceWindow]:
    """All windows of the trace, generated on the GPU (synth.DeviceStream)."""
    torch = _torch()
    st = synth.DeviceStream(trace, window_cycles, device)
    out = []
    while True:
        w = st.next()
        if w is None:
            break
        out.append(w)
    torch.cuda.synchronize()
    st.close()
    return out


def upload_trace(trace: synth.Trace, window_cycles: int, device: str = "cuda", threads: int = 0,
                 cap: int = 0) -> list[DeviceWindow]:
    """Generates the trace window by window on the host and copies each
    window into device memory through pinned staging buffers."""
    torch = _torch()
    st = synth.Stream(trace, window_cycles, threads)
    n_net, tpc, n_cycle = trace.n_net, trace.tpc, trace.n_cycle
    cap = cap or max(1 << 20, int(n_net * window_cycles * 0.12) + 4 * n_net)
    bufs = None
    out = []
    while True:
        if bufs is None or bufs[0].shape[0] < cap:
            bufs = (torch.empty(cap, dtype=torch.int64, pin_memory=True), np.empty(cap, np.uint8),
                    torch.empty(n_net + 1, dtype=torch.int64, pin_memory=True),
                    torch.empty(n_net, dtype=torch.int64, pin_memory=True),
                    torch.empty((cap + 15) // 16, dtype=torch.int32, pin_memory=True))
        times, values, net_off, net_base, packed = bufs
        try:
            r = st.next_into(times.numpy(), values, net_off.numpy(), net_base.numpy())
        except ValueError as e:  # buffers too small; nothing consumed
            cap = int(str(e).split(":")[1].split()[0]) + (1 << 16)
            continue
        if r is None:
            break
        n, t_lo, t_hi = r
        nw = (n + 15) // 16
        synth.synth_lib().synth_pack_values(values.ctypes.data, n, packed.data_ptr(), st.threads)
        w = DeviceWindow(t_lo // tpc, n_cycle if t_hi >= n_cycle * tpc else t_hi // tpc, t_lo, t_hi, n,
                         net_off.to(device, non_blocking=True), times[:max(n, 1)].to(device, non_blocking=True),
                         packed[:max(nw, 1)].to(device, non_blocking=True),
                         net_base.to(device, non_blocking=True))
        torch.cuda.current_stream().synchronize()  # staging buffers are reused
        out.append(w)
    return out


def cycle_total(c5: np.ndarray) -> np.ndarray:
    """Total per-cycle power from cycle5 rows (leakage + internal + switching,
    glitch included)."""
    return c5[..., 0, :] + c5[..., 1, :] + c5[..., 3, :]


def block_of_cells(n_cell: int, n_block: int) -> np.ndarray:
    return (np.arange(n_cell, dtype=np.int64) * n_block // n_cell).astype(np.int32)


def engine_labels(design, windows: list[DeviceWindow], n_block: int, **eng_kw):
    """Per-cycle total [n_period] and block powers [n_block, n_period] from
    the engine over all windows, with the walk's device time in seconds."""
    torch = _torch()
    with B200Power(design, **eng_kw) as eng:
        eng.set_cycle_groups(block_of_cells(design.n_cell, n_block), n_block)
        s = torch.cuda.ExternalStream(eng.stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for w in windows:
            w.push(eng)
        b.record(s)
        eng.sync()
        res = eng.fetch()
        G = eng.fetch_cycle_groups()
    return cycle_total(res.cycle5), cycle_total(G), a.elapsed_time(b) / 1e3


def engine_time(design, windows: list[DeviceWindow], c_lo: int, c_hi: int, **eng_kw):
    """The plain path over cycles [c_lo, c_hi) (windows aligned to them):
    per-cycle totals and device seconds."""
    torch = _torch()
    ws = [w for w in windows if w.c_lo >= c_lo and w.c_hi <= c_hi]
    with B200Power(design, **eng_kw) as eng:
        s = torch.cuda.ExternalStream(eng.stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for w in ws:
            w.push(eng)
        b.record(s)
        eng.sync()
        res = eng.fetch()
    return cycle_total(res.cycle5), a.elapsed_time(b) / 1e3


def engine_spot(design, windows: list[DeviceWindow], ranges: list[tuple[int, int]], **eng_kw):
    """The plain path over disjoint ascending cycle ranges only (audit and
    fallback): per-cycle totals (zero outside) and device seconds. Each
    window holding some of the ranges is walked once, over those ranges only
    (gtp_push_events_device_ranges)."""
    torch = _torch()
    with B200Power(design, **eng_kw) as eng:
        s = torch.cuda.ExternalStream(eng.stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for w in windows:
            mine = [(max(c0, w.c_lo), min(c1, w.c_hi)) for c0, c1 in ranges if max(c0, w.c_lo) < min(c1, w.c_hi)]
            if mine:
                w.push_ranges(eng, mine)
        b.record(s)
        eng.sync()
        res = eng.fetch()
    return cycle_total(res.cycle5), a.elapsed_time(b) / 1e3


def toggle_corr(windows, n_net: int, tpc: int, c_lo: int, c_hi: int, y) -> np.ndarray:
    """Pearson correlation over cycles [c_lo, c_hi) between each net's
    per-cycle toggle bit and y (a float32 device tensor of c_hi - c_lo)."""
    torch = _torch()
    dev = y.device
    cnt = torch.zeros(n_net, dtype=torch.int64, device=dev)
    sy = torch.zeros(n_net, dtype=torch.float64, device=dev)
    for w in windows:
        lo, hi = max(c_lo, w.c_lo), min(c_hi, w.c_hi)
        if lo < hi:
            px.net_toggle_stats(w.net_off, w.time, n_net, tpc, lo, hi, y[lo - c_lo:], cnt, sy)
    n = float(c_hi - c_lo)
    yd = y.double()
    my, sdy = yd.mean(), yd.std(unbiased=False)
    p = cnt.double() / n
    cov = sy / n - p * my
    den = torch.sqrt(torch.clamp(p * (1 - p), min=0)) * sdy
    corr = torch.where(den > 0, cov / torch.clamp(den, min=1e-300), torch.zeros_like(cov))
    return corr.cpu().numpy()


def select_nets(windows, n_net: int, tpc: int, c_lo: int, c_hi: int, Y: np.ndarray, k: int,
                exclude: tuple[int, ...] = ()) -> np.ndarray:
    """k nets: for each label column of Y [cycles, n_out] the ones with the
    largest |correlation| (k // n_out each), then by |correlation| with the
    first column (the total)."""
    torch = _torch()
    n_out = Y.shape[1]
    quota = k // n_out
    chosen: list[int] = []
    taken = np.zeros(n_net, bool)
    taken[list(exclude)] = True
    corr0 = None
    for o in range(n_out):
        y = torch.from_numpy(np.ascontiguousarray(Y[:, o], dtype=np.float32)).cuda()
        c = np.abs(toggle_corr(windows, n_net, tpc, c_lo, c_hi, y))
        if o == 0:
            corr0 = c
        c[taken] = -1
        top = np.argsort(-c, kind="stable")[:quota]
        top = top[c[top] > 0]
        chosen.extend(top.tolist())
        taken[top] = True
    c = corr0.copy()
    c[taken] = -1
    rest = np.argsort(-c, kind="stable")[: k - len(chosen)]
    chosen.extend(rest.tolist())
    return np.asarray(chosen[:k], dtype=np.int32)


def features(windows, sel: np.ndarray, tpc: int, c_lo: int, c_hi: int, out=None):
    """[c_hi - c_lo, len(sel)] BF16 toggle bits on the device."""
    torch = _torch()
    k = int(sel.shape[0])
    if out is None:
        out = torch.empty((c_hi - c_lo, k), dtype=torch.bfloat16, device="cuda")
    d_sel = torch.from_numpy(np.ascontiguousarray(sel, np.int32)).cuda()
    fill_toggle_bits(out, windows, d_sel, tpc, c_lo, c_hi)
    return out


def fill_toggle_bits(out, windows, d_sel, tpc: int, c_lo: int, c_hi: int, stream=None) -> None:
    """out[c - c_lo, k] = toggle bit of net d_sel[k] in cycle c for all c in
    [c_lo, c_hi): the windows' rows written densely in one launch per 64
    windows, rows of no window zeroed."""
    spans = []
    for w in windows:
        lo, hi = max(c_lo, w.c_lo), min(c_hi, w.c_hi)
        if lo < hi:
            spans.append((w.net_off, w.time, lo, hi))
    spans.sort(key=lambda s: s[2])
    done = c_lo
    for _, _, lo, hi in spans:
        if lo > done:
            out[done - c_lo:lo - c_lo].zero_()
        done = max(done, hi)
    if done < c_hi:
        out[done - c_lo:].zero_()
    px.toggle_bits_windows(spans, d_sel, tpc, c_lo, out, stream=stream)


def ridge_fit(X, Y, n_val: int, lams=(1e-3, 1e-2, 1e-1, 1.0, 10.0, 100.0, 1000.0)):
    """The method without the network: a ridge-regularised linear model on
    the same toggle bits (FP64, torch on the GPU), lambda picked on the last
    n_val training cycles, then refit on all of them. Returns
    (W [k+1, n_out], lambda)."""
    torch = _torch()
    Xd = torch.cat([X.double(), torch.ones((X.shape[0], 1), dtype=torch.float64, device=X.device)], 1)
    Yd = torch.as_tensor(Y, dtype=torch.float64, device=X.device)
    nv = max(1, min(n_val, Xd.shape[0] - 1))
    Xa, Ya, Xv, Yv = Xd[:-nv], Yd[:-nv], Xd[-nv:], Yd[-nv:]
    G = Xa.T @ Xa
    R = Xa.T @ Ya
    eye = torch.eye(G.shape[0], dtype=torch.float64, device=X.device)
    best = None
    for lam in lams:
        W = torch.linalg.solve(G + lam * eye, R)
        err = float(((Xv @ W - Yv) ** 2).mean())
        if best is None or err < best[0]:
            best = (err, lam)
    lam = best[1]
    W = torch.linalg.solve(Xd.T @ Xd + lam * eye, Xd.T @ Yd)
    return W, lam


def ridge_predict(W, X):
    torch = _torch()
    Xd = torch.cat([X.double(), torch.ones((X.shape[0], 1), dtype=torch.float64, device=X.device)], 1)
    return (Xd @ W).float()


def nrmse(pred: np.ndarray, ref: np.ndarray) -> float:
    """Per-cycle RMSE over the mean of the reference."""
    return float(np.sqrt(np.mean((pred - ref) ** 2)) / max(np.mean(ref), 1e-300))


def audit_ranges(c_lo: int, c_hi: int, frac: float, run: int, seed: int) -> list[tuple[int, int]]:
    """Disjoint ascending runs of `run` cycles covering about `frac` of
    [c_lo, c_hi)."""
    n_runs = max(1, int(round((c_hi - c_lo) * frac / run)))
    rng = np.random.default_rng(seed)
    slots = (c_hi - c_lo) // run
    pick = np.sort(rng.choice(slots, size=min(n_runs, slots), replace=False))
    return [(c_lo + int(s) * run, c_lo + int(s) * run + run) for s in pick]


def merge_ranges(cycles: np.ndarray, ranges: list[tuple[int, int]]) -> list[tuple[int, int]]:
    """Union of single cycles and ranges as disjoint ascending ranges."""
    m = set()
    for c0, c1 in ranges:
        m.update(range(c0, c1))
    m.update(int(c) for c in cycles)
    out: list[tuple[int, int]] = []
    for c in sorted(m):
        if out and out[-1][1] == c:
            out[-1] = (out[-1][0], c + 1)
        else:
            out.append((c, c + 1))
    return out


@dataclass
class ProxyReport:
    n_train: int
    n_infer: int
    nrmse_total: float
    nrmse_blocks: float
    total_power_error: float
    linear_nrmse_total: float
    linear_nrmse_blocks: float
    audit_nrmse_total: float
    ood_fraction: float
    audit_fraction: float
    spot_max_rel: float        # engine on spot ranges vs the full-trace labels
    plain_s: float
    proxy_s: float
    feature_s: float
    predict_s: float
    fallback_s: float
    train_s: float
    label_s: float
    select_s: float
    epochs: int
    best_epoch: int
    losses: list
    ridge_lambda: float

    @property
    def plain_cycles_per_s(self) -> float:
        return self.n_infer / self.plain_s

    @property
    def proxy_cycles_per_s(self) -> float:
        return self.n_infer / self.proxy_s

    @property
    def deployed_cycles_per_s(self) -> float:
        return self.n_infer / (self.proxy_s + self.fallback_s)


def run_flow(design, windows: list[DeviceWindow], tpc: int, n_train: int, n_block: int = 32, k: int = 4096,
             hidden: int = 512, batch: int = 1024, epochs: int = 40, lr: float = 1e-3, audit_frac: float = 0.01,
             audit_run: int = 10, seed: int = 1, exclude: tuple[int, ...] = (), weight_decay: float = 0.0,
             eval_every: int = 5, log=None) -> ProxyReport:
    """Labels, selection, training, inference, audit: the whole proxy flow
    over device-resident windows (aligned so that n_train is a window edge).
    The last 10% of the training cycles are held out: the network's
    parameters are kept from the epoch (checked every eval_every) with the
    lowest validation error, and the linear model's lambda is chosen there."""
    torch = _torch()
    say = log or (lambda *a: None)
    n_cycle = max(w.c_hi for w in windows)
    n_net = int(windows[0].net_off.shape[0] - 1)
    n_inf = n_cycle - n_train
    # 1. labels for every cycle (training targets, and the reference for the
    #    inference cycles' error)
    t0 = time.time()
    tot, blk, label_s = engine_labels(design, windows, n_block)
    Y = np.concatenate([tot[None, :], blk], 0).T[:n_cycle].astype(np.float32)  # [n_cycle, 1 + n_block]
    say(f"labels: {label_s:.3f} s device ({time.time() - t0:.1f} s wall)")
    # 2. selection on the training cycles
    t0 = time.time()
    sel = select_nets(windows, n_net, tpc, 0, n_train, Y[:n_train], k, exclude)
    select_s = time.time() - t0
    say(f"selection: {len(sel)} nets in {select_s:.1f} s")
    # 3. training
    X_tr = features(windows, sel, tpc, 0, n_train)
    n_val = max(batch, n_train // 10)
    n_fit = n_train - n_val
    Y_fit = torch.from_numpy(np.ascontiguousarray(Y[:n_fit])).cuda()
    Y_val = Y[n_fit:n_train]
    t0 = time.time()
    net = px.PowerProxy(n_in=len(sel), n_hidden=hidden, n_out=Y.shape[1], batch=batch, lr=lr, seed=seed,
                        weight_decay=weight_decay)
    net.set_training_data(X_tr[:n_fit], Y_fit)
    losses: list[float] = []
    best = (np.inf, None, 0)
    done = 0
    while done < epochs:
        n = min(eval_every, epochs - done)
        losses.extend(net.train(n).tolist())
        done += n
        pv = net.predict(X_tr[n_fit:]).cpu().numpy()
        err = float(np.mean([nrmse(pv[:, o], Y_val[:, o]) for o in range(Y.shape[1])]))
        if err < best[0]:
            best = (err, net.params_flat(), done)
    net.set_params_flat(best[1])
    train_s = time.time() - t0
    say(f"training: {epochs} epochs (kept epoch {best[2]}, validation {best[0]:.4f}), "
        f"loss {losses[0]:.4f} -> {losses[-1]:.4f}, {train_s:.1f} s")
    W_lin, lam = ridge_fit(X_tr, Y[:n_train], n_val)
    act_tr = X_tr.float().sum(1)
    a_lo, a_hi = float(act_tr.min()), float(act_tr.max())
    # 4. inference on the remaining cycles: features + network, device-timed
    X_inf = torch.empty((n_inf, len(sel)), dtype=torch.bfloat16, device="cuda")
    d_sel = torch.from_numpy(np.ascontiguousarray(sel, np.int32)).cuda()
    s = net.stream
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    with torch.cuda.stream(s):
        for _ in range(2):  # warm-up, then timed
            e0.record(s)
            fill_toggle_bits(X_inf, windows, d_sel, tpc, n_train, n_cycle, stream=s.cuda_stream)
            e1.record(s)
            pred = net.predict(X_inf, sync=False)
            e2.record(s)
            s.synchronize()
    feature_s = e0.elapsed_time(e1) / 1e3
    predict_s = e1.elapsed_time(e2) / 1e3
    P = pred.cpu().numpy()
    ref = Y[n_train:n_cycle]
    lin = ridge_predict(W_lin, X_inf).cpu().numpy()
    # 5. the plain path on the same cycles, timed alone (the throughput the
    #    proxy is compared with)
    _, plain_s = engine_time(design, windows, n_train, n_cycle)
    # 6. deployment: out-of-range cycles and an audit sample go to the engine
    act = X_inf.float().sum(1).cpu().numpy()
    ood = np.nonzero((act < a_lo) | (act > a_hi))[0] + n_train
    aud = audit_ranges(n_train, n_cycle, audit_frac, audit_run, seed)
    fb = merge_ranges(ood, aud)
    spot, fallback_s = engine_spot(design, windows, fb)
    in_aud = np.zeros(n_inf, bool)
    for c0, c1 in aud:
        in_aud[c0 - n_train:c1 - n_train] = True
    in_fb = np.zeros(n_cycle, bool)
    for c0, c1 in fb:
        in_fb[c0:c1] = True
    full_tot = Y[:, 0]
    spot_max_rel = float(np.max(np.abs(spot[:n_cycle][in_fb] - full_tot[in_fb]) / np.abs(full_tot[in_fb])))
    net.close()
    rb = [nrmse(P[:, 1 + b], ref[:, 1 + b]) for b in range(n_block)]
    lb = [nrmse(lin[:, 1 + b], ref[:, 1 + b]) for b in range(n_block)]
    return ProxyReport(
        n_train=n_train, n_infer=n_inf,
        nrmse_total=nrmse(P[:, 0], ref[:, 0]), nrmse_blocks=float(np.mean(rb)),
        total_power_error=float(abs(P[:, 0].sum() - ref[:, 0].sum()) / ref[:, 0].sum()),
        linear_nrmse_total=nrmse(lin[:, 0], ref[:, 0]), linear_nrmse_blocks=float(np.mean(lb)),
        audit_nrmse_total=nrmse(P[in_aud, 0], spot[n_train:n_cycle][in_aud]),
        ood_fraction=float(len(ood) / n_inf), audit_fraction=float(in_aud.mean()), spot_max_rel=spot_max_rel,
        plain_s=plain_s, proxy_s=feature_s + predict_s, feature_s=feature_s, predict_s=predict_s,
        fallback_s=fallback_s, train_s=train_s, label_s=label_s, select_s=select_s, epochs=epochs,
        best_epoch=best[2],
        losses=[float(x) for x in losses], ridge_lambda=float(lam))
