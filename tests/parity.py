"""Comparison of engine results against the FP64 oracle.

Integer counts (events walked, glitch classifications, toggles, related-pin
choices, per-cycle event and glitch counts) must match exactly. Powers are
compared with a relative tolerance of 1e-5 per value, with values below
1e-3 of their column's largest magnitude held to 1e-8 of that magnitude
instead (internal energies in Liberty tables can be negative, so a cell's
sum can cancel to near zero)."""
import numpy as np

RTOL = 1e-5
FLOOR = 1e-3


def close(name, got, ref, rtol=RTOL, floor=FLOOR):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    assert got.shape == ref.shape, (name, got.shape, ref.shape)
    if ref.size == 0:
        return 0.0
    scale = np.max(np.abs(ref), axis=0, keepdims=True) if ref.ndim > 1 else np.max(np.abs(ref))
    tol = rtol * np.maximum(np.abs(ref), floor * scale)
    err = np.abs(got - ref)
    bad = err > tol
    if bad.any():
        idx = np.argwhere(bad)[:5]
        raise AssertionError(f"{name}: {bad.sum()} values out of tolerance, e.g. "
                             + "; ".join(f"{tuple(i)} got {got[tuple(i)]:.9g} ref {ref[tuple(i)]:.9g}" for i in idx))
    big = np.abs(ref) > floor * scale
    return float(np.max(err[big] / np.abs(ref[big]))) if big.any() else 0.0


def compare(res, orc, check_counts=True):
    """Returns the max relative errors per quantity; raises on a mismatch."""
    out = {}
    if check_counts:
        c = res.counts
        for field in ("cell_events", "cell_glitches", "cell_half_toggles", "cell_related",
                      "cycle_events", "cycle_glitches"):
            g = getattr(c, field)
            r = getattr(orc, field)
            if not np.array_equal(g.astype(np.int64), r.astype(np.int64)):
                i = np.nonzero(g.astype(np.int64) != r.astype(np.int64))[0][:5]
                raise AssertionError(f"{field} differs at {i.tolist()}: got {g[i].tolist()} ref {r[i].tolist()}")
    out["cell"] = close("cell5", res.cell5, orc.cell5)
    out["cycle"] = close("cycle5", res.cycle5.T, orc.cycle5.T)
    out["totals"] = close("totals", res.totals, orc.totals)
    out["groups"] = close("groups", res.groups, orc.groups)
    return out
