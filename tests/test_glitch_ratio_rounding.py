"""The glitch scaling ratio's quotient in float.

The reference computes (pulse_width * 2.0) / sum_slew with a float pulse
width and a float slew sum in double and rounds the quotient to float
(power/PowerUtils.cc:285-294). The engine divides in float instead
(glitch_ratio_of in power_kernel.cu): the same bits, since rounding a
quotient of two floats first to double and then to float is innocuous
(53 >= 2 * 24 + 2 bits). Checked here on random operands over the ranges
the walk meets (pulse widths of one tick to a cycle, slews of femto- to
nanoseconds) and over whole binades, with numpy's IEEE float32 division as
the correctly rounded float quotient."""
import numpy as np


def _check(a, b):
    a = a.astype(np.float32)
    b = b.astype(np.float32)
    via_double = ((a.astype(np.float64) * 2.0) / b.astype(np.float64)).astype(np.float32)
    in_float = (a * np.float32(2.0)) / b
    assert np.array_equal(via_double.view(np.uint32), in_float.view(np.uint32))


def test_walk_ranges():
    rng = np.random.default_rng(1)
    n = 2_000_000
    pw = np.exp(rng.uniform(np.log(1e-13), np.log(1e-8), n))
    den = np.exp(rng.uniform(np.log(1e-15), np.log(1e-8), n))
    _check(pw, den)


def test_full_binades():
    rng = np.random.default_rng(2)
    n = 2_000_000
    # random significands, exponents over most of the normal float range
    a = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-60, 60, n))
    b = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-60, 60, n))
    _check(a, b)
