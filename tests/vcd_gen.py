"""Random VCD text for the reader tests: scalar, vector and real vars, ids
that look like values or times, repeated values, x/u/z values, vectors
written shorter than their width or starting with x, changes at time 0
through $dumpvars and changes of one id at one time."""
from __future__ import annotations

import numpy as np

_ID_CHARS = [chr(c) for c in range(33, 127)]


def _ids(rng: np.random.Generator, n: int) -> list[str]:
    out, seen = [], set()
    # ids that read like a time, a vector value or a real value when they
    # follow a vector or real token
    forced = ["#1", "b0", "b1x", "r", "0", "1a", "x", "zz", "#", "B10", "R2"]
    for f in forced[:n]:
        out.append(f)
        seen.add(f)
    while len(out) < n:
        k = int(rng.integers(1, 5))
        s = "".join(rng.choice(_ID_CHARS, k))
        if s not in seen:
            seen.add(s)
            out.append(s)
    return out


def make_vcd(rng: np.random.Generator, n_scalar: int = 30, n_vec: int = 10, n_real: int = 2, n_steps: int = 200,
             p_change: float = 0.3, width_max: int = 70) -> tuple[str, list[tuple[str, int]]]:
    """(VCD text, sources (id, bit) for every bit of every scalar and vector var)."""
    n = n_scalar + n_vec + n_real
    ids = _ids(rng, n)
    rng.shuffle(ids)
    kinds = ["s"] * n_scalar + ["v"] * n_vec + ["r"] * n_real
    widths = [1 if k == "s" else (int(rng.integers(2, width_max + 1)) if k == "v" else 64) for k in kinds]
    lines = ["$date today $end", "$version gen $end", "$timescale 1ps $end",
             "$scope module top $end", "$scope module dut $end"]
    for i, (k, w) in enumerate(zip(kinds, widths)):
        if k == "s":
            lines.append(f"$var wire 1 {ids[i]} s{i} $end")
        elif k == "v":
            lines.append(f"$var wire {w} {ids[i]} v{i} [{w - 1}:0] $end")
        else:
            lines.append(f"$var real 64 {ids[i]} r{i} $end")
    # an alias: a second var on the first id
    lines.append(f"$var wire {widths[0]} {ids[0]} alias0 $end")
    lines += ["$upscope $end", "$upscope $end", "$enddefinitions $end"]
    prev = {}

    def change(i):
        k = kinds[i]
        if k == "s":
            c = str(rng.choice(list("0101xzuXZU"))) if rng.random() < 0.8 else prev.get(i, "0")
            prev[i] = c
            return f"{c}{ids[i]}"
        if k == "r":
            return f"r{rng.uniform(-5, 5):.3f} {ids[i]}"
        w = widths[i]
        if rng.random() < 0.1:
            bits = str(rng.choice(list("xzuXZ"))) + "".join(rng.choice(list("01x"), int(rng.integers(0, w))))
        elif rng.random() < 0.15 and i in prev:
            bits = prev[i]
        else:
            bits = "".join(rng.choice(list("01"), int(rng.integers(1, w + 1))))
        prev[i] = bits
        return f"{'b' if rng.random() < 0.8 else 'B'}{bits} {ids[i]}"

    body = ["#0", "$dumpvars"]
    for i in range(n):
        if rng.random() < 0.6:
            body.append(change(i))
    body.append("$end")
    t = 0
    for _ in range(n_steps):
        t += int(rng.integers(1, 50))
        body.append(f"#{t}")
        for i in range(n):
            if rng.random() < p_change:
                body.append(change(i))
                if rng.random() < 0.03:        # a second change at the same time
                    body.append(change(i))
    sep = rng.choice(["\n", "\n", " ", "\r\n", "\t"], len(body))
    text = "\n".join(lines) + "\n" + "".join(b + str(s) for b, s in zip(body, sep)) + "\n"
    sources = []
    for i, (k, w) in enumerate(zip(kinds, widths)):
        if k == "s":
            sources.append((ids[i], 0))
        elif k == "v":
            sources += [(ids[i], b) for b in range(w)]
    return text, sources
