"""Throughput benchmark of the time-based power walk on one or more B200s.

Workload: the flat synthetic sky130hd design (200k cells, 10k cycles of
2 ns at 1 ps ticks, per-net toggle probability U[0.05, 0.3], glitch pulses
p=0.05 of 5-100 ps); ~4e8 net events. One step = one full evaluation of the
trace: clear accumulators, walk every cell over every cycle, finalize the
per-cell and per-cycle outputs.

  value : net events / s with the event CSR resident in HBM
  e2e   : the same through the public host API (B200Power.read_power_activities
          from pinned host memory + fetch of per-cell/per-cycle results)

Multi-GPU (torchrun, --gpus N): every rank evaluates its own trace of the same
design (independent seeds); no collective is needed (weak scaling).
--impl reference times the CPU restatement of the reference CPU path (FP32,
static thread split as power/Power.cc:227-386) on the host cores over a
bounded sample of cells.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

def metric_name(cells: int, cycles: int) -> str:
    """The flat workload's metric, named by its size (200k cells x 10k cycles by default)."""
    def k(n: int) -> str:
        return f"{n // 1000}k" if n % 1000 == 0 else str(n)
    return f"net events/s (time-based power walk, flat synthetic {k(cells)} cells x {k(cycles)} cycles)"
UNIT = "events/s"


def workload_name(args) -> str:
    """The default workload's description, the same on the engine's line and the reference arm's."""
    return (f"flat synthetic sky130hd {args.cells} cells x {args.cycles} cycles "
            "(2 ns, 1 ps ticks, toggle U[0.05,0.3], glitch p=0.05)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cells", type=int, default=200_000)
    ap.add_argument("--cycles", type=int, default=10_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity leg (the timed configuration's outputs against the FP64 oracle)")
    ap.add_argument("--cycles-per-tile", type=int, default=0)
    ap.add_argument("--e2e-split", default="ramp", choices=["ramp", "even"],
                    help="e2e windows: 'ramp' grows them by --e2e-ramp each (a short first copy, then each "
                         "copy hides behind the walk of the window before), 'even' cuts equal windows")
    ap.add_argument("--e2e-ramp", type=float, default=1.25,
                    help="growth of each e2e window over the one before (ramp split)")
    ap.add_argument("--e2e-windows", type=int, default=12,
                    help="the e2e leg pushes the trace from pinned host memory as this many windows "
                         "(with their context), so that each window's copy overlaps the previous walk")
    ap.add_argument("--gates-per-block", type=int, default=0)
    ap.add_argument("--threads-per-block", type=int, default=0)
    ap.add_argument("--split-events", type=int, default=0,
                    help="density split: events per thread and tile above which a cell is walked by "
                         "several threads (0: the engine's default, -1: off)")
    ap.add_argument("--separate-kernels", action="store_true",
                    help="flat workload: evaluate with the two unfused kernels (a thread per pin event for "
                         "the dynamic energies, a thread per cell and tile for the leakage), the reference's "
                         "-disable_fusion baseline, instead of the fused walk")
    ap.add_argument("--warp-walk", action="store_true",
                    help="walk cells of up to 4 pins with one warp each, 32 events at a time (default: one "
                         "thread per cell and tile)")
    ap.add_argument("--no-clock-runs", action="store_true",
                    help="walk periodic clock pins edge by edge instead of as runs of whole cycles")
    ap.add_argument("--workload", default="flat", choices=["flat", "proxy", "batch", "stream", "gemm"],
                    help="flat: the plain walk (default); proxy: the learned per-cycle power proxy "
                         "against the plain walk on a phased-unit trace; batch: 64 uneven traces x "
                         "3 corners in persistent batched launches")
    ap.add_argument("--stream-cells", type=int, default=2_000_000)
    ap.add_argument("--stream-cycles", type=int, default=20_000)
    ap.add_argument("--stream-window", type=int, default=512)
    ap.add_argument("--stream-e2e-gb", type=float, default=6.0,
                    help="pinned host bytes of windows replayed through the host API (a bounded sample)")
    ap.add_argument("--batch-traces", type=int, default=64)
    ap.add_argument("--batch-window", type=int, default=2048)
    ap.add_argument("--batch-max-cells", type=int, default=500_000)
    ap.add_argument("--batch-max-cycles", type=int, default=50_000)
    ap.add_argument("--proxy-cells", type=int, default=1_000_000)
    ap.add_argument("--proxy-cycles", type=int, default=100_000)
    ap.add_argument("--proxy-train", type=int, default=20_000)
    ap.add_argument("--proxy-window", type=int, default=2_000)
    ap.add_argument("--proxy-epochs", type=int, default=40)
    ap.add_argument("--proxy-inputs", type=int, default=4096)
    ap.add_argument("--gemm-rows", type=int, default=80_000,
                    help="gemm: rows (cycles) of the proxy's inference, and of each single GEMM timed")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(pg, values, device):
    """Each value's maximum over the ranks (the slowest rank's time); pg is
    torch.distributed or None for one process."""
    if pg is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return t.tolist()


def workload(args, rank: int):
    from gtpower_b200 import synth
    spec = synth.FlatSpec(n_cell=args.cells, n_cycle=args.cycles, seed=20261203 + 1)
    design, info = synth.flat_design(spec)
    trace = synth.Trace(design, info, synth.TraceSpec(), seed=20261203 + 1 + 1000 * rank)
    return design, info, trace


def e2e_cuts(cycles: int, windows: int, ramp: float) -> np.ndarray:
    """Cycle boundaries [0, c1, ..., cycles] of the e2e windows: `windows`
    windows whose sizes grow by `ramp` each (a short first copy; each later
    copy hides behind the walk of the window before), rounded to whole
    cycles, empty windows dropped."""
    sizes = ramp ** np.arange(windows)
    cuts = np.concatenate([[0], np.round(np.cumsum(sizes) / sizes.sum() * cycles)]).astype(np.int64)
    return np.unique(cuts)


def algorithmic_bytes(design, n_event: int) -> int:
    """8 B tick + 2 bits per net event, CSR offsets, 24 B of attributes per
    pin, the LUT floats, and 20 B of outputs per cell and per cycle."""
    return int(8 * n_event + (n_event + 3) // 4 + 8 * (design.n_net + 1) + 24 * design.n_pin
               + 4 * int(design.lib.lut_pool.shape[0]) + 20 * design.n_cell + 20 * design.n_period)


def pin_events(design, net_off: np.ndarray) -> int:
    cnt = np.diff(net_off)
    p = design.pin_net
    return int(cnt[p[p >= 0]].sum())


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self) -> dict:
        self._stop.set()
        if self._t:
            self._t.join(timeout=6)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_peak_tensor():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def run_proxy(args):
    """Learned per-cycle power proxy against the plain walk: phased-unit
    trace (16 sticky phases, p_stay 0.99, 32 net units), engine labels on the
    first proxy-train cycles, 4096 inputs chosen by correlation, MLP
    4096-512-512-33 trained with the tcgen05 kernels, inference on the rest."""
    import torch
    from gtpower_b200 import proxy_flow as pf
    from gtpower_b200 import synth
    torch.cuda.set_device(0)
    t0 = time.time()
    spec = synth.FlatSpec(n_cell=args.proxy_cells, n_cycle=args.proxy_cycles, seed=20261203 + 4)
    design, info = synth.flat_design(spec)
    tspec = synth.TraceSpec(mode=3, lo=0.02, hi=0.12, n_phase=16, p_stay=0.99, n_unit=32, act_sigma=1.0,
                            glitch_p=0.05)
    trace = synth.Trace(design, info, tspec, seed=20261203 + 4)
    wins = pf.generate_on_device(trace, args.proxy_window)
    n_event = sum(w.n_event for w in wins)
    gen_s = time.time() - t0
    print(f"# trace: {n_event} events in {len(wins)} windows, {gen_s:.1f} s", file=sys.stderr, flush=True)
    sampler = ClockSampler(0)
    sampler.start()
    rep = pf.run_flow(design, wins, info["tpc"], n_train=args.proxy_train, n_block=32, k=args.proxy_inputs,
                      hidden=512, batch=1024, epochs=args.proxy_epochs, lr=1e-3, audit_frac=0.01,
                      audit_run=10, seed=5, exclude=(info["clock_net"],),
                      log=lambda m: print("# " + m, file=sys.stderr, flush=True))
    clocks = sampler.stop()
    op = (33 + 7) // 8 * 8
    flops = 2.0 * rep.n_infer * (args.proxy_inputs * 512 + 512 * 512 + 512 * op)
    peak, kind = measured_peak_tensor()
    achieved = flops / rep.predict_s / 1e12
    line = {
        "metric": "per-cycle waveform cycles/s: learned proxy vs plain walk "
                  f"({args.proxy_cells} cells x {args.proxy_cycles} cycles, {rep.n_infer} inferred)",
        "value": rep.proxy_cycles_per_s, "unit": "cycles/s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": rep.proxy_s * 1e3, "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
        "config": {"workload": f"phased-unit synthetic {args.proxy_cells} cells x {args.proxy_cycles} cycles, "
                               f"train {args.proxy_train}, MLP {args.proxy_inputs}-512-512-33",
                   "n_event": n_event, "windows": len(wins), "generation_s": gen_s},
        "plain_cycles_per_s": rep.plain_cycles_per_s,
        "speedup_vs_plain": rep.proxy_cycles_per_s / rep.plain_cycles_per_s,
        "deployed_cycles_per_s": rep.deployed_cycles_per_s,
        "nrmse_total": rep.nrmse_total, "nrmse_blocks_mean": rep.nrmse_blocks,
        "total_power_error": rep.total_power_error,
        "linear_nrmse_total": rep.linear_nrmse_total, "linear_nrmse_blocks_mean": rep.linear_nrmse_blocks,
        "audit_nrmse_total": rep.audit_nrmse_total, "audit_fraction": rep.audit_fraction,
        "ood_fraction": rep.ood_fraction, "spot_vs_full_max_rel": rep.spot_max_rel,
        "times_s": {"plain": rep.plain_s, "features": rep.feature_s, "predict": rep.predict_s,
                    "fallback": rep.fallback_s, "train": rep.train_s, "labels": rep.label_s,
                    "select": rep.select_s},
        "training": {"epochs": rep.epochs, "loss_first": rep.losses[0], "loss_last": rep.losses[-1],
                     "ridge_lambda": rep.ridge_lambda},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": f"{kind} (MEASURED_PEAKS.json bf16_tflops)" if kind == "measured" else "fallback",
                     "kernel": "gemm_kernel (3 layers, inference)"},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_gemm(args):
    """The proxy's inference on the tcgen05 GEMM, on its own: the MLP
    4096-512-512-33 over --gemm-rows cycles of random toggle bits (the
    gtp_proxy_predict path: three GEMMs with fused bias/ReLU and BF16
    activations), and each layer's shape as one GEMM with an FP32 output
    (gtp_bf16_gemm). Device time by CUDA events on the launching streams,
    after warm-up."""
    import torch
    from gtpower_b200 import proxy as px
    torch.cuda.set_device(0)
    m, k_in, h, n_out = args.gemm_rows, args.proxy_inputs, 512, 33
    g = torch.Generator(device="cuda").manual_seed(20261203 + 5)
    x = (torch.rand(m, k_in, device="cuda", generator=g) < 0.2).to(torch.bfloat16)
    net = px.PowerProxy(n_in=k_in, n_hidden=h, n_out=n_out)
    s = net.stream
    out = torch.empty((m, n_out), dtype=torch.float32, device="cuda")
    sampler = ClockSampler(0)
    sampler.start()
    for _ in range(args.warmup):
        net.predict(x, out=out)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for a, b in evs:
        a.record(s)
        net.predict(x, out=out, sync=False)
        b.record(s)
    s.synchronize()
    pred_ms = [a.elapsed_time(b) for a, b in evs]
    op = (n_out + 7) // 8 * 8
    flops = 2.0 * m * (k_in * h + h * h + h * op)
    layers = {}
    for name, (kk, nn) in {"layer1": (k_in, h), "layer2": (h, h), "layer3": (h, op)}.items():
        a_ = torch.randn(m, kk, device="cuda", generator=g).to(torch.bfloat16)
        b_ = torch.randn(nn, kk, device="cuda", generator=g).to(torch.bfloat16)
        for _ in range(args.warmup):
            px.bf16_gemm(a_, b_)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            px.bf16_gemm(a_, b_)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        layers[name] = {"m": m, "n": nn, "k": kk, "ms": ms, "tflops": 2.0 * m * nn * kk / ms / 1e9}
        del a_, b_
    clocks = sampler.stop()
    net.close()
    peak, kind = measured_peak_tensor()
    ms = float(np.median(pred_ms))
    achieved = flops / ms / 1e9
    line = {
        "metric": f"proxy inference TFLOP/s (MLP {k_in}-512-512-33 over {m} cycles, tcgen05 BF16 GEMMs)",
        "value": achieved, "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "bf16",
        "data": "synthetic", "config": {"workload": f"random toggle bits {m} x {k_in} (p=0.2), random weights"},
        "cycles_per_s": m / (ms / 1e3), "single_gemm_fp32_out": layers,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": f"{kind} (MEASURED_PEAKS.json bf16_tflops)" if kind == "measured" else "fallback",
                     "kernel": "gemm_kernel (3 layers, inference)"},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def h2d_peak_gbs(nbytes: int = 1 << 30) -> float:
    """Pinned host -> device copy bandwidth on this box (best of 5)."""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    best = 0.0
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        d.copy_(h, non_blocking=True)
        b.record()
        b.synchronize()
        best = max(best, nbytes / (a.elapsed_time(b) / 1e3) / 1e9)
    del h, d
    return best


def run_stream(args):
    """Skewed trace streamed through HBM: 2M cells, 20k cycles, per-net
    rates Zipf(1.2) scaled to mean 0.1, per-cycle burst factor lognormal
    (sigma 1.5, mean 1), glitch p=0.1. Windows of --stream-window cycles (with
    their head/tail context) are generated on the GPU; value = net events/s of
    the walk on device-resident windows; e2e = the first windows (up to
    --stream-e2e-gb) replayed from pinned host memory through the host API,
    whose copies overlap the previous window's walk."""
    import torch
    from gtpower_b200 import B200Power, batch, synth
    torch.cuda.set_device(0)
    log = lambda m: print("# " + m, file=sys.stderr, flush=True)
    t0 = time.time()
    design, info = synth.flat_design(synth.FlatSpec(n_cell=args.stream_cells, n_cycle=args.stream_cycles,
                                                    seed=20261203 + 2))
    spec = synth.TraceSpec(mode=1, zipf_alpha=1.2, rate_mean=0.1, burst_sigma=1.5, glitch_p=0.1)
    build_s = time.time() - t0
    W = args.stream_window
    # autotune the block shape on the first window
    st = synth.DeviceStream(synth.Trace(design, info, spec, seed=20261203 + 2), W)
    w0 = st.next()
    st.close()
    torch.cuda.synchronize()
    best, table = batch.tune([design], [w0], log=log)
    log(f"autotuner: {best}")
    # device-resident windows, timed walk; warm-up: the first window three
    # times on the timed context (its tables grow to size), each undone by a reset
    eng = B200Power(design, split_events=args.split_events, **best.engine_kw())
    s = torch.cuda.ExternalStream(eng.stream)
    for _ in range(3):
        w0.push(eng)
        eng.sync()
        eng.reset()
    del w0
    st = synth.DeviceStream(synth.Trace(design, info, spec, seed=20261203 + 2), W)
    total_ev, walk_s, gen_s, n_win, max_win = 0, 0.0, 0.0, 0, 0
    split_items = []
    host_wins, host_bytes = [], 0
    walk_times = []
    sampler = ClockSampler(0)
    sampler.start()
    while True:
        g0 = time.time()
        w = st.next()
        torch.cuda.synchronize()
        gen_s += time.time() - g0
        if w is None:
            break
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        w.push(eng)
        b.record(s)
        eng.sync()
        walk_s += a.elapsed_time(b) / 1e3
        walk_times.append(a.elapsed_time(b) / 1e3)
        split_items.append(eng.walk_items())
        total_ev += w.n_event
        max_win = max(max_win, w.n_event)
        n_win += 1
        wb = w.n_event * 8 + w.packed.numel() * 4 + w.net_off.numel() * 8 + w.net_base.numel() * 8
        if host_bytes + wb <= args.stream_e2e_gb * 1e9:
            host_wins.append((w.n_event, w.t_lo, w.t_hi, w.net_off.cpu().pin_memory(), w.time[:max(1, w.n_event)].cpu().pin_memory(),
                              w.packed.cpu().pin_memory(), w.net_base.cpu().pin_memory()))
            host_bytes += wb
        del w
    clocks = sampler.stop()
    res = eng.fetch()
    eng.close()
    st.close()
    torch.cuda.empty_cache()
    # e2e: host windows through gtp_push_events (double-buffered copies)
    from gtpower_b200.design import Events
    h2d_gbs = h2d_peak_gbs()
    eng = B200Power(design, split_events=args.split_events, **best.engine_kw())
    s = torch.cuda.ExternalStream(eng.stream)
    evs = [Events(no.numpy(), tm.numpy(), pk.numpy().view(np.uint32), net_base=nb.numpy(), t_lo=lo, t_hi=hi)
           for (n, lo, hi, no, tm, pk, nb) in host_wins]
    e2e_ev = sum(h[0] for h in host_wins)
    # one untimed pass first: the context sizes its event slots and walk
    # scratch to the largest window on first use
    for ev in evs:
        eng.read_power_activities(ev)
    eng.sync()
    eng.reset()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for ev in evs:
        eng.read_power_activities(ev)
    b.record(s)
    eng.sync()
    e2e_s = a.elapsed_time(b) / 1e3
    eng.close()
    peak, kind = measured_peak_hbm()
    ab = algorithmic_bytes(design, total_ev)
    achieved = ab / walk_s / 1e9
    line = {
        "metric": f"net events/s, streamed skewed trace ({args.stream_cells} cells x {args.stream_cycles} cycles)",
        "value": total_ev / walk_s, "unit": "events/s", "n_gpus": 1, "steps": n_win, "warmup": 3,
        "ms_per_step": walk_s * 1e3 / max(1, n_win), "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"flat synthetic {args.stream_cells} cells x {args.stream_cycles} cycles, "
                               "Zipf(1.2) net rates mean 0.1, lognormal(1.5) per-cycle bursts, glitch p=0.1; "
                               f"windows of {W} cycles generated on the GPU",
                   "n_event": total_ev, "windows": n_win, "max_window_events": max_win,
                   "max_window_gb": max_win * 8.25 / 1e9, "autotuned_shape": best.__dict__,
                   "design_build_s": build_s, "generation_s": gen_s,
                   "density_split": {"split_events": args.split_events,
                                     "walk_threads_per_tile_max": max(split_items) if split_items else 0,
                                     "cells": design.n_cell}},
        "e2e": {"value": e2e_ev / e2e_s, "unit": "events/s", "windows": len(host_wins),
                "same_windows_device_resident_events_per_s": e2e_ev / max(1e-12, sum(walk_times[:len(host_wins)])),
                "h2d_bytes_per_step": int(host_bytes / max(1, len(host_wins))), "d2h_bytes_per_step": 0,
                "sample": f"first {len(host_wins)} windows ({host_bytes / 1e9:.2f} GB pinned) via gtp_push_events, "
                          "after one untimed pass over them",
                "h2d_link_gbs_measured": h2d_gbs,
                "h2d_frac": (host_bytes / e2e_s / 1e9) / h2d_gbs},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": kind, "algorithmic_bytes": ab,
                     "kernel": "power_walk_kernel"},
        "clocks": clocks,
        "totals_w": {"leakage": float(res.totals[0]), "internal": float(res.totals[1]),
                     "switching": float(res.totals[3])},
    }
    print(json.dumps(line), flush=True)


def run_batch(args):
    """64 synthetic traces of uneven size (cells log-uniform in [1e4, 5e5],
    cycles log-uniform in [1e3, 5e4], toggle U[0.05, 0.3], glitch p=0.05),
    3 corners (leakage and internal tables x 0.8 / 1.0 / 1.3) folded from one
    walk, in persistent batched launches window by window; block shape from
    the autotuner. Windows are generated on the GPU before each timed push."""
    import torch
    from gtpower_b200 import B200Power, batch, synth
    torch.cuda.set_device(0)
    rng = np.random.default_rng(20261203 + 3)
    n_tr = args.batch_traces
    cells = np.exp(rng.uniform(np.log(1e4), np.log(args.batch_max_cells), n_tr)).astype(np.int64)
    cycles = np.exp(rng.uniform(np.log(1e3), np.log(args.batch_max_cycles), n_tr)).astype(np.int64)
    t0 = time.time()
    designs, traces = [], []
    for i in range(n_tr):
        d, info = synth.flat_design(synth.FlatSpec(n_cell=int(cells[i]), n_cycle=int(cycles[i]),
                                                   seed=20261203 + 3 + i))
        designs.append(d)
        traces.append(synth.Trace(d, info, synth.TraceSpec(), seed=20261203 + 3 + 1000 + i))
    build_s = time.time() - t0
    W = args.batch_window
    log = lambda m: print("# " + m, file=sys.stderr, flush=True)
    log(f"{n_tr} designs built in {build_s:.1f} s; cells {int(cells.sum())}, max cycles {int(cycles.max())}")
    # autotune on the first windows of every 4th trace
    sample = list(range(0, n_tr, 4))
    sw = []
    for i in sample:
        st = synth.DeviceStream(traces[i], W)
        sw.append(st.next())
        st.close()
    torch.cuda.synchronize()
    best, table = batch.tune([designs[i] for i in sample], sw, log=log)
    del sw
    torch.cuda.empty_cache()
    log(f"autotuner: {best}")
    engines = [B200Power(d, **best.engine_kw()) for d in designs]
    streams = [synth.DeviceStream(tr, W) for tr in traces]
    bp = batch.BatchPower(engines)
    s = torch.cuda.ExternalStream(bp.stream)
    bufs = [None] * n_tr
    total_ev = 0
    walk_s = 0.0
    gen_s = 0.0
    waves = 0
    seq_s = None
    seq_ev = 0
    batch_wave0_s = None
    sampler = ClockSampler(0)
    sampler.start()
    while True:
        g0 = time.time()
        wins = [st.next(out=bufs[i]) if st is not None else None for i, st in enumerate(streams)]
        for i, w in enumerate(wins):
            if w is None and streams[i] is not None:
                streams[i].close()
                streams[i] = None
            elif w is not None:
                bufs[i] = w
        torch.cuda.synchronize()
        gen_s += time.time() - g0
        if all(w is None for w in wins):
            break
        if waves == 0:  # the same windows one design at a time, for comparison
            seq_eng = [B200Power(d, **best.engine_kw()) for d in designs]
            batch.run_sequential(seq_eng, wins)          # warm-up
            for e in seq_eng:
                e.reset()
            seq_s = batch.run_sequential(seq_eng, wins)
            seq_ev = sum(w.n_event for w in wins if w is not None)
            # the same windows batched, warm: separate engines, a first push
            # (buffers, graph capture), reset, then the timed replay
            with batch.BatchPower(seq_eng) as bw:
                for e in seq_eng:
                    e.reset()
                bw.push(wins)
                bw.sync()
                for e in seq_eng:
                    e.reset()
                sw_ = torch.cuda.ExternalStream(bw.stream)
                a0, b0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a0.record(sw_)
                bw.push(wins)
                b0.record(sw_)
                bw.sync()
                batch_wave0_s = a0.elapsed_time(b0) / 1e3
            for e in seq_eng:
                e.close()
            # warm-up of the timed batch: its buffers and graph come with its
            # first push; the first wave three times, each undone by a reset
            for _ in range(3):
                bp.push(wins)
                bp.sync()
                for e in engines:
                    e.reset()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        bp.push(wins)
        b.record(s)
        bp.sync()
        dt = a.elapsed_time(b) / 1e3
        walk_s += dt
        total_ev += sum(w.n_event for w in wins if w is not None)
        waves += 1
    clocks = sampler.stop()
    stats = bp.stats()
    # corners folded from the one walk
    f0 = time.time()
    corner_totals = []
    for e in engines:
        r = e.fetch()
        corner_totals.append([float(np.sum(batch.fold_corner(r, ls, is_).totals[[0, 1, 3]]))
                              for ls, is_ in batch.CORNERS])
    fold_s = time.time() - f0
    bp.close()
    peak, kind = measured_peak_hbm()
    line = {
        "metric": f"net events/s, batched persistent walk ({n_tr} uneven traces x 3 corners)",
        "value": total_ev / walk_s, "unit": "events/s", "n_gpus": 1, "steps": waves, "warmup": 3,
        "ms_per_step": walk_s * 1e3 / max(1, waves), "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{n_tr} flat synthetic traces, cells log-uniform [1e4, {args.batch_max_cells}], "
                               f"cycles log-uniform [1e3, {args.batch_max_cycles}], toggle U[0.05,0.3], glitch 0.05; "
                               f"corners x0.8/x1.0/x1.3 folded from one walk; windows of {W} cycles",
                   "n_event_total": total_ev, "cells_total": int(cells.sum()),
                   "cell_cycles_total": int((cells * cycles).sum()), "waves": waves,
                   "autotuned_shape": best.__dict__,
                   "autotune_ms": {f"{c.cycles_per_tile}/{c.threads_per_block}/{c.gates_per_block}": t * 1e3
                                   for c, t in table},
                   "design_build_s": build_s, "generation_s": gen_s},
        "corner_events_per_s": 3 * total_ev / walk_s,
        "cell_cycles_per_s": float((cells * cycles).sum()) / walk_s,
        "first_wave": {"events": seq_ev,
                       "one_design_at_a_time_events_per_s": seq_ev / seq_s if seq_s else None,
                       "batched_events_per_s": seq_ev / batch_wave0_s if batch_wave0_s else None,
                       "batched_speedup": (seq_s / batch_wave0_s) if (seq_s and batch_wave0_s) else None,
                       "note": "both warm: each side pushed the wave once before the timed push"},
        "batch_stats": stats, "corner_fold_s": fold_s,
        "roofline": {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                     "traffic": None, "peak_source": kind, "kernel": "power_walk_batch_kernel"},
        "clocks": clocks,
    }
    ab = 8.25 * total_ev / walk_s / 1e9
    line["roofline"]["achieved"] = ab
    line["roofline"]["frac"] = ab / peak
    print(json.dumps(line), flush=True)


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(design, ev, total_events: int):
    """The FP32 restatement of the reference CPU path (power/Power.cc:227-386:
    static cell split over a thread pool, per-thread per-cycle arrays) over
    every cell of the trace, on all host threads: a measured duration of the
    whole workload, not an extrapolation."""
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    r = orc.run(design, ev, fp32=True, threads=threads, outputs=False)
    return {"value": total_events / max(r.seconds, 1e-9), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"the whole workload: all {design.n_cell} cells, {total_events} net events, "
                      f"{r.seconds:.2f} s on {threads} threads (per-pin slews and arc delays "
                      "precomputed, where the reference queries its timing graph per event)",
            "seconds": r.seconds}


def _rel_errors(got: np.ndarray, ref: np.ndarray, floor: float = 1e-3) -> dict:
    """Largest relative error of got against ref per column (quantity), over
    the values above floor x the column's largest magnitude, and the largest
    error of the rest relative to that magnitude (sums that cancel to near
    zero are held to the column scale)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    out = {}
    names = ["leakage", "internal", "glitch_internal", "switching", "glitch_switching"]
    for q in range(ref.shape[1]):
        g, r = got[:, q], ref[:, q]
        scale = float(np.max(np.abs(r))) if r.size else 0.0
        big = np.abs(r) > floor * scale
        rel = float(np.max(np.abs(g[big] - r[big]) / np.abs(r[big]))) if big.any() else 0.0
        small = float(np.max(np.abs(g[~big] - r[~big])) / scale) if (~big).any() and scale > 0 else 0.0
        out[names[q]] = {"max_rel": rel, "small_max_abs_over_scale": small}
    return out


def parity_leg(design, ev, results: dict, counts_res, threads: int) -> dict:
    """The engine's outputs of the timed configuration against an FP64
    re-evaluation of the reference CPU path (the oracle) over the whole
    trace: integer counts bit for bit, and the relative error of every
    reported quantity per cell, per cycle and in the totals."""
    from oracle import oracle as orc
    ref = orc.run(design, ev, fp32=False, threads=threads)
    # cell5 columns: internal, glitch internal, switching, glitch switching, leakage
    # (internal and switching without glitch); in the oracle's order of cycle5
    perm = [4, 0, 1, 2, 3]
    out = {"oracle": f"FP64 restatement of the reference CPU path over all {design.n_cell} cells",
           "oracle_seconds": ref.seconds, "tolerance": "1e-5 relative (values under 1e-3 of their "
           "column's largest magnitude: 1e-8 of it)"}
    ok = True
    for name, res in results.items():
        cell = _rel_errors(res.cell5[:, perm], ref.cell5[:, perm])
        cyc = _rel_errors(res.cycle5.T, ref.cycle5.T)
        tot = {k: float(abs(res.totals[q] - ref.totals[q]) / max(abs(ref.totals[q]), 1e-300))
               for q, k in enumerate(["leakage", "internal", "glitch_internal", "switching", "glitch_switching"])}
        worst = max([v["max_rel"] for v in cell.values()] + [v["max_rel"] for v in cyc.values()]
                    + list(tot.values()))
        worst_small = max([v["small_max_abs_over_scale"] for v in cell.values()]
                          + [v["small_max_abs_over_scale"] for v in cyc.values()])
        ok = ok and worst <= 1e-5 and worst_small <= 1e-8
        out[name] = {"cell": cell, "cycle": cyc, "totals": tot, "max_rel": worst}
    if counts_res is not None:
        c = counts_res.counts
        fields = ("cell_events", "cell_glitches", "cell_half_toggles", "cell_related",
                  "cycle_events", "cycle_glitches")
        mism = {f: int(np.count_nonzero(getattr(c, f).astype(np.int64) != getattr(ref, f).astype(np.int64)))
                for f in fields}
        out["counts_exact"] = all(v == 0 for v in mism.values()) and c.dropped == ref.dropped
        out["count_mismatches"] = mism
        out["pin_events_counted"] = int(c.cell_events.astype(np.int64).sum())
        out["glitch_events_counted"] = int(c.cell_glitches.astype(np.int64).sum())
        ok = ok and out["counts_exact"]
    out["pass"] = bool(ok)
    return out


def run_reference(args, rank, world):
    """The reference arm: the FP32 restatement of the reference CPU path
    (the reference's own build needs Tcl, SWIG, flex, bison, Eigen3 and CUDD,
    which this image lacks) over every cell of the same trace in each timed
    step, on all host threads. Warm-up steps walk a small cell sample."""
    if rank != 0:
        return
    design, info, trace = workload(args, 0)
    ev = trace.full()
    total_events = ev.n_event
    tpe = pin_events(design, ev.net_off)
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(11)
    warm = rng.permutation(design.n_cell)[:max(threads * 4, 2000)].astype(np.int32)
    for _ in range(args.warmup):
        orc.run(design, ev, fp32=True, threads=threads, cells=warm, outputs=False)
    secs = []
    for _ in range(args.steps):
        r = orc.run(design, ev, fp32=True, threads=threads, outputs=False)
        secs.append(r.seconds)
    ms = float(np.mean(secs)) * 1e3
    value = total_events / (ms / 1e3)
    line = {"metric": metric_name(args.cells, args.cycles), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload_name(args), "n_event": total_events, "pin_events": tpe},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"the whole workload each timed step: all {design.n_cell} cells, "
                                       f"{total_events} net events; warm-up steps walk {warm.shape[0]} cells; "
                                       "per-pin slews and arc delays precomputed (the reference queries "
                                       "its timing graph per event)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.workload == "proxy":
        if rank == 0:
            run_proxy(args)
        return
    if args.workload == "batch":
        if rank == 0:
            run_batch(args)
        return
    if args.workload == "stream":
        if rank == 0:
            run_stream(args)
        return
    if args.workload == "gemm":
        if rank == 0:
            run_gemm(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    from gtpower_b200 import B200Power
    from gtpower_b200.design import Events

    design, info, trace = workload(args, rank)
    t0 = time.time()
    ev = trace.full()
    gen_s = time.time() - t0
    n_event = ev.n_event
    tpe = pin_events(design, ev.net_off)

    # pinned host copies (e2e leg) and device copies (value leg)
    h_off = torch.from_numpy(ev.net_off).pin_memory()
    h_t = torch.from_numpy(ev.time).pin_memory()
    h_v = torch.from_numpy(ev.packed.view(np.int32)).pin_memory()
    pinned = Events(h_off.numpy(), h_t.numpy(), h_v.numpy().view(np.uint32))
    d_off = h_off.cuda()
    d_t = h_t.cuda()
    d_v = h_v.cuda()
    # e2e windows: the same trace cut at cycle boundaries, each with its
    # context, in pinned host memory (prepared before timing, like the trace)
    from gtpower_b200 import synth as _synth
    e2e_wins = []
    h2d = 0
    if args.e2e_windows > 1:
        if args.e2e_split == "ramp":
            from gtpower_b200 import windows as _windows
            tpc = design.ticks_per_cycle
            cuts = e2e_cuts(args.cycles, args.e2e_windows, args.e2e_ramp)
            wins_src = [_windows.make_window(ev, tpc, int(cuts[k]) * tpc,
                                             int(cuts[k + 1]) * tpc if k + 2 < len(cuts) else np.iinfo(np.int64).max)
                        for k in range(len(cuts) - 1)]
        else:
            st = _synth.Stream(trace, (args.cycles + args.e2e_windows - 1) // args.e2e_windows)
            wins_src = []
            while True:
                w = st.next(n_event + 4 * design.n_net)
                if w is None:
                    break
                wins_src.append(w)
        for w in wins_src:
            pt = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
                  for a in (w.net_off, w.time, w.packed.view(np.int32), w.net_base)]
            e2e_wins.append((pt, Events(pt[0].numpy(), pt[1].numpy(), pt[2].numpy().view(np.uint32),
                                        net_base=pt[3].numpy(), t_lo=w.t_lo, t_hi=w.t_hi)))
            h2d += 8 * (design.n_net + 1) + 8 * w.n_event + 4 * ((w.n_event + 15) // 16) + 8 * design.n_net
    else:
        e2e_wins = [(None, pinned)]
        h2d = 8 * (design.n_net + 1) + 8 * n_event + 4 * ((n_event + 15) // 16)

    eng = B200Power(design, device=local, cycles_per_tile=args.cycles_per_tile,
                    gates_per_block=args.gates_per_block, threads_per_block=args.threads_per_block,
                    clock_runs=not args.no_clock_runs, split_events=args.split_events,
                    separate_kernels=args.separate_kernels, warp_walk=args.warp_walk)
    stream = torch.cuda.ExternalStream(eng.stream)

    def device_step():
        eng.reset()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        eng.push_device(n_event, d_off.data_ptr(), d_t.data_ptr(), d_v.data_ptr())
        ev1.record(stream)
        return ev0, ev1

    # per step: tile_first, glitch_pw, pclk, work_keys (then the library's
    # radix sort), split_count (then the library's scan), the walk (one pin
    # bucket here), finalize_cells, finalize_cycles; with the separate
    # kernels: tile_first, glitch_pw, sep_net_range, sep_cell_count (then the
    # library's scan), sep_dyn, power_leak (one pin bucket), the two finalize
    launches_per_step = 8
    from gtpower_b200 import _abi
    import ctypes as C

    def finalize_device():
        # finalize kernels only (results stay on the device for the value leg)
        _abi.check(_abi.lib().gtp_finalize(eng.ctx), eng.ctx)

    for _ in range(args.warmup):
        device_step()
        finalize_device()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    kern = []
    for _ in range(args.steps):
        kern.append(device_step())
        finalize_device()
    s1.record(stream)
    torch.cuda.synchronize()
    step_ms = s0.elapsed_time(s1) / args.steps
    walk_ms = float(np.mean([a.elapsed_time(b) for a, b in kern]))

    # e2e leg: host pinned buffers through the public API, results back to host
    e2e_ms_list = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.reset()
        for _, w in e2e_wins:
            eng.read_power_activities(w)
        res = eng.fetch()
        b.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e_ms_list.append(a.elapsed_time(b))
    clocks = sampler.stop()
    e2e_ms = float(np.mean(e2e_ms_list))

    # max over ranks
    step_ms, e2e_ms, walk_ms = max_over_ranks(pg, [step_ms, e2e_ms, walk_ms], "cuda")

    d2h = 4 * 5 * design.n_cell + 4 * 5 * eng.n_period + 8 * 5 * 6 + 4
    b_alg = algorithmic_bytes(design, n_event)
    peak, peak_kind = measured_peak_hbm()
    achieved = b_alg / (walk_ms / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic_power_walk.json")
    if os.path.exists(prof):
        try:
            with open(prof) as f:
                tj = json.load(f)
            traffic = int(tj["bytes_per_launch_scaled"])
        except Exception:
            traffic = None

    # results of the timed configuration for the parity leg: the
    # device-resident single window and the host-pushed windows of the e2e leg
    res_e2e = res
    device_step()
    res_dev = eng.fetch()
    counts_res = None
    if rank == 0 and not args.no_parity:
        with B200Power(design, device=local, cycles_per_tile=args.cycles_per_tile,
                       gates_per_block=args.gates_per_block, threads_per_block=args.threads_per_block,
                       clock_runs=not args.no_clock_runs, split_events=args.split_events,
                       separate_kernels=args.separate_kernels, warp_walk=args.warp_walk,
                       collect_counts=True) as ceng:
            ceng.push_device(n_event, d_off.data_ptr(), d_t.data_ptr(), d_v.data_ptr())
            counts_res = ceng.fetch(counts=True)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(design, ev, n_event)
        cpu.pop("seconds", None)
    parity = None
    if rank == 0 and not args.no_parity:
        parity = parity_leg(design, ev, {"device_resident": res_dev, f"e2e_{len(e2e_wins)}_windows": res_e2e},
                            counts_res, os.cpu_count() or 1)

    if rank == 0:
        line = {
            "metric": metric_name(args.cells, args.cycles),
            "value": world * n_event / (step_ms / 1e3),
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(args),
                       "n_event": n_event, "pin_events": tpe, "n_cell": design.n_cell,
                       "n_pin": design.n_pin, "n_net": design.n_net, "n_period": eng.n_period,
                       "cell_cycles_per_s": world * design.n_cell * eng.n_period / (step_ms / 1e3),
                       "l2": "inputs larger than L2 (event CSR %.2f GB)" % (h2d / 1e9),
                       "walk_ms": walk_ms, "generation_s": gen_s,
                       "clock_pins": ("edge by edge" if args.no_clock_runs or args.separate_kernels
                                      else "runs of whole cycles when periodic"),
                       "evaluation": ("separate kernels: a thread per pin event (dynamic), then a thread per "
                                      "cell and tile (leakage)" if args.separate_kernels
                                      else "fused walk, cells of up to 4 pins one warp each" if args.warp_walk
                                      else "fused walk, one thread per cell and tile"),
                       "parallelism": f"weak: {world} independent traces" if world > 1 else "1 GPU"},
            "e2e": {"value": world * n_event / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                    "windows": len(e2e_wins), "split": args.e2e_split if len(e2e_wins) > 1 else "one window"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None if args.separate_kernels else traffic,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                         "algorithmic_bytes_per_launch": b_alg,
                         "kernel": "sep_dyn_kernel + power_leak_kernel" if args.separate_kernels else "power_walk_kernel"},
            "cpu_baseline": cpu,
            "parity": parity,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
            "totals_w": {"leakage": float(res.totals[0]), "internal": float(res.totals[1]),
                         "switching": float(res.totals[3])},
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
