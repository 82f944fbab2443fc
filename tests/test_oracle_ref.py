"""The oracle's helpers against the reference's own functions.

tests/golden/ref_vectors.npz holds inputs and outputs of the reference's
table interpolation (liberty/TableModel.cc Table1/Table2::findValue,
findValueIndex), cycle index (power/PowerUtils.cc clkedWaveformIdx), toggle
and rise counts (getNToggle, getNRise) and glitch scaling ratio
(getTimeBasedGlitchScalingRatioH), produced by those functions compiled from
the reference sources (oracle/Makefile target `ref`;
tests/golden/make_ref_vectors.py). The oracle must reproduce every output
bit for bit in its FP32 mode; in its FP64 mode the interpolated table
values must round to the reference's float results.

When the compiled reference helpers are present (oracle/_ref/libref.so,
built where the reference sources are), fresh random inputs are checked
against them directly as well."""
import os

import numpy as np
import pytest

from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
VEC = os.path.join(HERE, "golden", "ref_vectors.npz")


@pytest.fixture(scope="module")
def vec():
    return dict(np.load(VEC))


def _oracle_table(order, n1, n2, a1, a2, v, x1, x2, fp32):
    L = orc.lib()
    return L.oracle_table_value(order, int(n1), a1.ctypes.data, int(n2), a2.ctypes.data, v.ctypes.data,
                                float(x1), float(x2), 1 if fp32 else 0)


@pytest.mark.parametrize("order", [1, 2])
def test_table_interpolation_matches_reference(vec, order):
    p = f"t{order}_"
    n = vec[p + "y"].shape[0]
    bad32, bad64 = [], []
    for i in range(n):
        args = (order, vec[p + "n1"][i], vec[p + "n2"][i], vec[p + "a1"][i], vec[p + "a2"][i], vec[p + "v"][i],
                vec[p + "x1"][i], vec[p + "x2"][i])
        y = vec[p + "y"][i]
        y32 = np.float32(_oracle_table(*args, fp32=True))
        y64 = _oracle_table(*args, fp32=False)
        if y32.view(np.uint32) != y.view(np.uint32):
            bad32.append(i)
        if np.float32(y64).view(np.uint32) != y.view(np.uint32):
            bad64.append(i)
    assert not bad32, [(i, vec[p + "y"][i]) for i in bad32[:5]]
    assert not bad64, bad64[:5]


@pytest.mark.parametrize("order", [1, 2])
def test_axis_bisection_matches_reference(vec, order):
    p = f"t{order}_"
    L = orc.lib()
    got = np.array([L.oracle_find_value_index(vec[p + "a1"][i].ctypes.data, int(vec[p + "n1"][i]),
                                              float(vec[p + "x1"][i])) for i in range(vec[p + "idx"].shape[0])])
    assert np.array_equal(got, vec[p + "idx"])


def test_cycle_index_matches_reference(vec):
    L = orc.lib()
    got = np.array([L.oracle_cycle_of(int(t), float(ts), float(per))
                    for t, ts, per in zip(vec["cyc_t"], vec["cyc_ts"], vec["cyc_period"])], np.int64)
    assert np.array_equal(got, vec["cyc_idx"])


def test_toggle_and_rise_match_reference(vec):
    L = orc.lib()
    tg = np.array([L.oracle_n_toggle(int(a), int(b)) for a, b in zip(vec["tg_prev"], vec["tg_cur"])], np.float32)
    rs = np.array([L.oracle_n_rise(int(a), int(b)) for a, b in zip(vec["tg_prev"], vec["tg_cur"])], np.float32)
    assert np.array_equal(tg, vec["tg_toggle"])
    assert np.array_equal(rs, vec["tg_rise"])


def test_glitch_ratio_matches_reference(vec):
    L = orc.lib()
    got32 = np.array([L.oracle_glitch_ratio(int(w), float(ts), float(a), float(b), 1)
                      for w, ts, a, b in zip(vec["gl_w"], vec["gl_ts"], vec["gl_sr"], vec["gl_sf"])], np.float32)
    assert np.array_equal(got32.view(np.uint32), vec["gl_ratio"].view(np.uint32))
    got64 = np.array([L.oracle_glitch_ratio(int(w), float(ts), float(a), float(b), 0)
                      for w, ts, a, b in zip(vec["gl_w"], vec["gl_ts"], vec["gl_sr"], vec["gl_sf"])])
    # FP64 mode keeps the pulse width and the ratio in double: within float rounding
    assert np.allclose(got64, vec["gl_ratio"], rtol=1e-6, atol=0)


def test_fresh_inputs_against_compiled_reference():
    """Live check against the compiled reference helpers, on inputs other
    than the committed vectors."""
    R = orc.ref_lib()
    if R is None:
        pytest.skip("reference helpers not compiled here (oracle/_ref/libref.so)")
    import importlib.util
    spec = importlib.util.spec_from_file_location("mrv", os.path.join(HERE, "golden", "make_ref_vectors.py"))
    mrv = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mrv)
    rng = np.random.default_rng(7)
    for order in (1, 2):
        n1, n2, a1, a2, v, x1, x2 = mrv.table_cases(rng, 500, order)
        for i in range(500):
            if order == 1:
                y = R.ref_table1(a1[i].ctypes.data, int(n1[i]), v[i].ctypes.data, float(x1[i]))
            else:
                y = R.ref_table2(a1[i].ctypes.data, int(n1[i]), a2[i].ctypes.data, int(n2[i]), v[i].ctypes.data,
                                 float(x1[i]), float(x2[i]))
            got = np.float32(_oracle_table(order, n1[i], n2[i], a1[i], a2[i], v[i], x1[i], x2[i], fp32=True))
            assert got.view(np.uint32) == np.float32(y).view(np.uint32), (order, i)
    L = orc.lib()
    for t in rng.integers(0, 1 << 42, 300):
        for ts in (1e-12, 1e-9, 1e-15):
            per = np.float32(np.exp(rng.uniform(np.log(1e-10), np.log(1e-6))))
            assert L.oracle_cycle_of(int(t), ts, float(per)) == R.ref_clked_waveform_idx(int(t), float(np.float32(ts)),
                                                                                          float(per))
