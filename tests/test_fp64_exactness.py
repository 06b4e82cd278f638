"""The FP64 identities the device fast paths rely on, checked on the host in IEEE double.

* round_half_away(x) == trunc(x + copysign(0.5 - 2^-54, x)) for every double x (the prediction's
  rounding, glc_device.cuh predict_from / half_away_bias);
* for integers |y| < 2^51 and predictions |x| <= 2^51: fabs(y - trunc(x + bias)) computed in
  float64 equals |y - round_half_away(x)| exactly (abs_resid_fp64, used by the split search, the
  merge pass, the fit's max error and the batch kernels);
* for x >= -0.25 the constant addend 0.5 - 2^-54 gives the same rounding (the split search's band
  loops).
The exact reference is Python's integer and Fraction arithmetic.
"""
import math
from fractions import Fraction

import numpy as np

BIAS = np.float64(0.5) - np.float64(2.0) ** -54  # 0.5 - 2^-54, exactly representable


def round_half_away_exact(x: float) -> int:
    f = Fraction(x)
    n = math.floor(abs(f) + Fraction(1, 2))
    return n if f >= 0 else -n


def trunc_biased(x: np.float64) -> np.float64:
    return np.trunc(x + np.copysign(BIAS, x))


def _samples(rng, count):
    xs = []
    # ties and near-ties at small and large magnitudes
    for k in list(range(-40, 41)) + [2 ** 20 + 3, 2 ** 40 + 7, 2 ** 50 + 1, -(2 ** 50) - 5]:
        t = np.float64(k) + np.float64(0.5)
        xs += [t, np.nextafter(t, np.inf), np.nextafter(t, -np.inf)]
    xs += list(rng.uniform(-1e6, 1e6, count))
    xs += list(rng.uniform(-(2.0 ** 51), 2.0 ** 51, count))
    xs += list(np.float64(rng.integers(-(2 ** 51), 2 ** 51, count)) + rng.uniform(-1, 1, count))
    return [np.float64(x) for x in xs]


def test_rounding_identity():
    rng = np.random.default_rng(7)
    for x in _samples(rng, 4000):
        assert int(trunc_biased(x)) == round_half_away_exact(float(x)), x


def test_constant_addend_for_nonnegative_predictions():
    rng = np.random.default_rng(8)
    xs = [x for x in _samples(rng, 4000) if x >= -0.25] + list(np.float64(rng.uniform(-0.25, 0.0, 500)))
    for x in xs:
        assert int(np.trunc(x + BIAS)) == round_half_away_exact(float(x)), x


def test_fp64_residual_is_exact_inside_bounds():
    rng = np.random.default_rng(9)
    lim = 2 ** 51
    ys = list(rng.integers(-lim + 1, lim, 3000)) + [lim - 1, -lim + 1, 0, 1, -1]
    xs = _samples(rng, 1000)
    for i, y in enumerate(ys):
        x = xs[i % len(xs)]
        if abs(float(x)) > 2.0 ** 51:
            continue
        got = np.abs(np.float64(y) - trunc_biased(x))
        want = abs(int(y) - round_half_away_exact(float(x)))
        assert int(got) == want and float(got) == want, (y, x)
