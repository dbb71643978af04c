"""The Jacobi sweep loop's test `resid / resid0 > 0.5` (Poisson::vcycle_relax,
poisson.cpp:88-130) is evaluated on the device as `resid > 0.5 * resid0`
whenever resid0 >= 2^-1021 (`above_half` in relax_brick.cuh), and with the
division otherwise.  The two agree for every pair of doubles there: 0.5 is
a double and rounding is monotonic, so they could differ only for an exact
quotient in (0.5, 0.5 + 2^-54], which two doubles cannot produce.  Checked
here in IEEE double arithmetic (numpy) on random pairs over the whole
exponent range and on the neighbours of 0.5 * resid0 where a disagreement
would have to sit."""

import numpy as np


def above_half(r, r0):
    with np.errstate(all="ignore"):
        return np.where(r0 >= 2.0 ** -1021, r > 0.5 * r0, r / r0 > 0.5)


def by_division(r, r0):
    with np.errstate(all="ignore"):
        return r / r0 > 0.5


def test_comparison_equals_division():
    rng = np.random.default_rng(20261204)
    n = 1_000_000
    r0 = np.exp(rng.uniform(-700.0, 700.0, n))
    half = 0.5 * r0
    cases = [half, np.nextafter(half, np.inf), np.nextafter(half, -np.inf),
             np.nextafter(np.nextafter(half, np.inf), np.inf),
             half * (1.0 + rng.uniform(-1e-15, 1e-15, n)),
             np.exp(rng.uniform(-700.0, 700.0, n))]
    for r in cases:
        assert np.array_equal(above_half(r, r0), by_division(r, r0))


def test_special_values():
    vals = np.array([0.0, -0.0, 5e-324, 2.0 ** -1022, 2.0 ** -1021, 1.0, np.inf, np.nan, 1e308])
    r, r0 = np.meshgrid(vals, vals)
    assert np.array_equal(above_half(r, r0), by_division(r, r0))
