"""The library's result-file writers against a restatement of the
reference's writers.

oracle/writers_ref.cpp keeps the reference's data flow for these files: per
instance, internal and switching power with the glitch part folded in as
float PowerResult fields (power/cuda/CudaPower.cu:3011-3019), the row's
regular part as folded - glitch and its total as the float sum of the five
columns (:3134-3165), numbers through std::ostream, and the per-cycle file's
five sections (include/sta/PowerClass.hh:123-149). Given the same
per-instance values, the files gtp_write_cell_power and
gtp_write_per_cycle_waveform write must equal its files byte for byte."""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_build", "writers_ref")


@pytest.fixture(scope="module")
def writers_ref():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "_build/writers_ref"], check=True)
    return REF


def _ref_files(tmp, cell5, cycle5, top, sep, names, types):
    blob = struct.pack("<iq", cell5.shape[0], cycle5.shape[1])
    blob += np.ascontiguousarray(cell5, np.float32).tobytes() + np.ascontiguousarray(cycle5, np.float32).tobytes()
    for s in [top, sep] + list(names) + list(types):
        blob += s.encode() + b"\0"
    inp = tmp / "in.bin"
    inp.write_bytes(blob)
    subprocess.run([REF, str(inp), str(tmp / "ref_cell.txt"), str(tmp / "ref_cycle.txt")], check=True)
    return (tmp / "ref_cell.txt").read_bytes(), (tmp / "ref_cycle.txt").read_bytes()


def _values(rng, shape):
    """Powers as the engine produces them, plus the edge values a float
    column can hold (zero, negative sums, subnormals, large and tiny values)."""
    v = (rng.standard_normal(shape) * 10.0 ** rng.integers(-14, -2, shape)).astype(np.float32)
    flat = v.reshape(-1)
    edge = np.array([0.0, -0.0, 1e-45, -3e-39, 1e-30, 123456.7, 1e38, -2.5e-7, 1.0, 0.1], np.float32)
    flat[:edge.size] = edge
    return v


@pytest.mark.parametrize("sep", ["\t", ", "])
def test_cell_and_cycle_files_match_reference_writers(tmp_path, writers_ref, sep):
    from gtpower_b200 import _abi
    from gtpower_b200.design import Design
    from gtpower_b200.power import PowerResult, write_cell_power
    from gtpower_b200 import synth
    rng = np.random.default_rng(3)
    d, _ = synth.flat_design(synth.FlatSpec(n_cell=700, n_cycle=5, seed=9))
    d.cell_names = [f"u_core/blk{i % 7}/cell_{i}" for i in range(d.n_cell)]
    cell5 = _values(rng, (d.n_cell, 5))
    cycle5 = _values(rng, (5, 37))
    write_cell_power(str(tmp_path / "cell.txt"), d, cell5, sep)
    PowerResult(waveforms=cycle5).print_per_cycle_results(str(tmp_path / "cycle.txt"), "synth_top", sep)
    types = [d.lib.names[t] for t in d.cell_type]
    rc, ry = _ref_files(tmp_path, cell5, cycle5, "synth_top", sep, d.cell_names, types)
    assert (tmp_path / "cell.txt").read_bytes() == rc
    assert (tmp_path / "cycle.txt").read_bytes() == ry


def test_gcd_files_match_reference_writers(tmp_path, writers_ref):
    """The GCD example's oracle results written by the Python mirror's
    print_cell_res / print_per_cycle_results."""
    from gtpower_b200 import tape
    from gtpower_b200.power import B200Power, Results
    here = os.path.join(ROOT, "tests", "golden")
    d, ev, meta = tape.load(os.path.join(here, "gcd_tape.npz"))
    g = np.load(os.path.join(here, "gcd_oracle.npz"))
    eng = B200Power.__new__(B200Power)      # the writers need no device
    eng.design = d
    eng.ctx = None
    eng.n_period = d.n_period
    eng._results = Results(g["cell5"].astype(np.float32), g["cycle5"].astype(np.float32), g["totals"], g["groups"])
    eng.print_cell_res(str(tmp_path / "cuda_cell_power.txt"))
    total = eng.power()[0]
    total.print_per_cycle_results(str(tmp_path / "cuda_per_cycle_waveform.txt"), d.top_name)
    names = d.cell_names or [f"inst{i}" for i in range(d.n_cell)]
    types = [d.lib.names[t] for t in d.cell_type]
    rc, ry = _ref_files(tmp_path, eng._results.cell5, eng._results.cycle5, d.top_name, "\t", names, types)
    assert (tmp_path / "cuda_cell_power.txt").read_bytes() == rc
    assert (tmp_path / "cuda_per_cycle_waveform.txt").read_bytes() == ry
    text = rc.decode().splitlines()
    assert len(text) == d.n_cell + 1 and text[0].startswith("cell\tInternal_Power")


def test_writer_rejects_bad_arguments(tmp_path):
    from gtpower_b200 import _abi
    L = _abi.lib()
    assert L.gtp_write_cell_power(str(tmp_path / "x").encode(), 3, None, None, None, None, None) == _abi.GTP_EINVAL
    assert L.gtp_write_per_cycle_waveform(b"/nonexistent-dir/x.txt", 0, None, b"t", None) == _abi.GTP_GENERAL_ERROR
