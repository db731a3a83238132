"""The split engine's slicing rule (CPU): the s int8 slices of a scaled value x in
(-1, 1) are its leading base-128 digits, truncated toward zero, each carrying the
sign of x.  The device kernels take them from one integer, trunc(x 2^(7s)), by
shifts and masks; this checks that rule against the defining recursion
(a_t = trunc(128 x_t), x_{t+1} = 128 x_t - a_t) and the truncation bound
|x - sum_t a_t 128^-(t+1)| < 128^-s that the engine's error analysis uses."""
import math

import numpy as np
import pytest


def digits_recursive(x, s):
    out = []
    for _ in range(s):
        v = x * 128.0
        a = math.trunc(v)
        out.append(int(a))
        x = v - a
    return out


def digits_integer(x, s):
    y = math.ldexp(x, 7 * s)
    n = int(y) if abs(y) < 9.0e18 else 0
    a = abs(n)
    sign = -1 if n < 0 else 1
    return [sign * ((a >> (7 * (s - 1 - t))) & 127) for t in range(s)]


@pytest.mark.parametrize("s", range(1, 9))
def test_integer_digits_equal_the_recursion(s):
    rng = np.random.default_rng(100 + s)
    xs = np.concatenate([rng.uniform(-1, 1, 4000), rng.uniform(-1, 1, 500) * 1e-9,
                         [0.0, -0.0, 0.5, -0.5, 1 - 2.0 ** -53, -(1 - 2.0 ** -53), 2.0 ** -7, -(2.0 ** -14)]])
    for x in xs:
        x = float(x)
        d = digits_integer(x, s)
        assert d == digits_recursive(x, s)
        assert all(-127 <= v <= 127 for v in d)
        approx = sum(v * 128.0 ** -(t + 1) for t, v in enumerate(d))
        assert abs(x - approx) < 128.0 ** -s
