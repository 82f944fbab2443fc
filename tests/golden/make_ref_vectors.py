"""Generates tests/golden/ref_vectors.npz: inputs and outputs of the
reference's own helpers, compiled from its sources by oracle/Makefile
(target `ref`), so that the oracle's restatement can be checked against
them where the reference sources are absent.

    python tests/golden/make_ref_vectors.py --ref <path of the reference checkout>

Covers (file:line within the reference):
  Table1::findValue, Table2::findValue   liberty/TableModel.cc:858-880, 1011-1060
  findValueIndex                         liberty/TableModel.cc:1467-1489
  clkedWaveformIdx                       power/PowerUtils.cc:27-32
  getNRise, getNToggle                   power/PowerUtils.cc:213-255
  getTimeBasedGlitchScalingRatioH        power/PowerUtils.cc:285-294
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

MAXN = 8


def table_cases(rng: np.random.Generator, n: int, order: int):
    """Random NLDM-like tables: strictly increasing axes (slews 1 ps..2 ns,
    caps 0.1 fF..0.5 pF), signed energies, lookups inside, outside and on
    the axis points."""
    n1 = rng.integers(1, MAXN + 1, n).astype(np.int32)
    n2 = (rng.integers(1, MAXN + 1, n) if order == 2 else np.ones(n)).astype(np.int32)
    a1 = np.zeros((n, MAXN), np.float32)
    a2 = np.zeros((n, MAXN), np.float32)
    vals = np.zeros((n, MAXN * MAXN), np.float32)
    x1 = np.zeros(n, np.float32)
    x2 = np.zeros(n, np.float32)
    for i in range(n):
        for a, k, lo, hi, x in ((a1, n1[i], 1e-12, 2e-9, x1), (a2, n2[i], 1e-16, 5e-13, x2)):
            ax = np.sort(np.exp(rng.uniform(np.log(lo), np.log(hi), k))).astype(np.float32)
            while k > 1 and np.any(np.diff(ax) <= 0):
                ax = np.sort(np.exp(rng.uniform(np.log(lo), np.log(hi), k))).astype(np.float32)
            a[i, :k] = ax
            mode = rng.integers(0, 5)
            if mode == 0:      # on an axis point
                x[i] = ax[rng.integers(0, k)]
            elif mode == 1:    # below the axis (extrapolation)
                x[i] = np.float32(ax[0] * rng.uniform(0.0, 1.0))
            elif mode == 2:    # above the axis (extrapolation)
                x[i] = np.float32(ax[-1] * rng.uniform(1.0, 3.0))
            else:              # inside
                x[i] = np.float32(np.exp(rng.uniform(np.log(ax[0]), np.log(ax[-1]))))
        m = n1[i] * n2[i]
        vals[i, :m] = (rng.standard_normal(m) * 1e-14 + rng.uniform(-2e-15, 8e-15)).astype(np.float32)
    return n1, n2, a1, a2, vals, x1, x2


def generate(seed: int = 20261203, n_tab: int = 1500, n_cyc: int = 2000, n_gl: int = 2000) -> dict:
    from oracle import oracle as orc
    R = orc.ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libref.so is missing: build it with --ref")
    rng = np.random.default_rng(seed)
    out = {}
    for order in (1, 2):
        n1, n2, a1, a2, vals, x1, x2 = table_cases(rng, n_tab, order)
        y = np.zeros(n_tab, np.float32)
        idx = np.zeros(n_tab, np.int64)
        for i in range(n_tab):
            if order == 1:
                y[i] = R.ref_table1(a1[i].ctypes.data, int(n1[i]), vals[i].ctypes.data, float(x1[i]))
            else:
                y[i] = R.ref_table2(a1[i].ctypes.data, int(n1[i]), a2[i].ctypes.data, int(n2[i]),
                                    vals[i].ctypes.data, float(x1[i]), float(x2[i]))
            idx[i] = R.ref_find_value_index(a1[i].ctypes.data, int(n1[i]), float(x1[i]))
        p = f"t{order}_"
        out.update({p + "n1": n1, p + "n2": n2, p + "a1": a1, p + "a2": a2, p + "v": vals, p + "x1": x1,
                    p + "x2": x2, p + "y": y, p + "idx": idx})
    # cycle index: timescales of common VCD units, float periods
    ts = rng.choice(np.array([1e-15, 1e-12, 1e-11, 1e-10, 1e-9, 1e-6]), n_cyc)
    per = np.exp(rng.uniform(np.log(1e-10), np.log(1e-6), n_cyc)).astype(np.float32)
    per[: n_cyc // 8] = np.float32(2e-9)
    per[n_cyc // 8: n_cyc // 4] = np.float32(5e-9)
    t = rng.integers(0, 1 << 40, n_cyc, dtype=np.int64)
    cyc = np.array([R.ref_clked_waveform_idx(int(t[i]), float(np.float32(ts[i])), float(per[i]))
                    for i in range(n_cyc)], np.int64)
    out.update({"cyc_t": t, "cyc_ts": ts, "cyc_period": per, "cyc_idx": cyc})
    # glitch ratio: pulse widths in ticks, ps ticks, slews 0 and 5 ps..1 ns
    w = rng.integers(1, 3000, n_gl, dtype=np.int64)
    gts = np.full(n_gl, 1e-12)
    sr = np.exp(rng.uniform(np.log(5e-12), np.log(1e-9), n_gl)).astype(np.float32)
    sf = np.exp(rng.uniform(np.log(5e-12), np.log(1e-9), n_gl)).astype(np.float32)
    sr[:50] = 0
    sf[:50] = 0
    pulse = (w.astype(np.float64) * gts).astype(np.float32)       # VcdEventTime * timeScale -> float
    ssum = (sr + sf).astype(np.float32)                             # SlewVal sum in float
    g = np.array([R.ref_glitch_ratio(float(pulse[i]), float(ssum[i])) for i in range(n_gl)], np.float32)
    out.update({"gl_w": w, "gl_ts": gts, "gl_sr": sr, "gl_sf": sf, "gl_ratio": g})
    # toggle and rise over every pair of values 0, 1, X (2), Z (3)
    pv, cv = np.meshgrid(np.arange(4), np.arange(4), indexing="ij")
    out["tg_prev"] = pv.ravel().astype(np.int32)
    out["tg_cur"] = cv.ravel().astype(np.int32)
    out["tg_toggle"] = np.array([R.ref_n_toggle(int(a), int(b)) for a, b in zip(pv.ravel(), cv.ravel())], np.float32)
    out["tg_rise"] = np.array([R.ref_n_rise(int(a), int(b)) for a, b in zip(pv.ravel(), cv.ravel())], np.float32)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the reference checkout (sources are read in place)")
    ap.add_argument("--out", default=os.path.join(HERE, "ref_vectors.npz"))
    a = ap.parse_args()
    from oracle import oracle as orc
    orc.build_ref(a.ref)
    vec = generate()
    np.savez_compressed(a.out, **vec)
    print(f"wrote {a.out}: " + ", ".join(f"{k}{list(v.shape)}" for k, v in vec.items()))


if __name__ == "__main__":
    main()
