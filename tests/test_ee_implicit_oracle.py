"""The opt-in backward-Euler f00 e-e step (OSHUN_FLAG_IMPLICIT_EE) in the C
checker, against the reference's explicit scheme (Explicit_EC_FP::loop,
OSHUN-1/def-FokkerPlanck.cpp:590-625, restated in the oracle):

* consistency: one step of length D differs from the explicit RK4 step
  (fine substeps) by O(D^2), so the difference drops ~4x per halving of D;
* conservation: over 5 steps of D = 2 (4 explicit substeps each) the
  number and energy moments move as the explicit scheme moves them;
* stability: 10 steps of D = 200 (400 explicit substeps each) keep f00
  positive and finite, keep the number to 1e-4 and land within 5 % of the
  explicit run (0.2 % with 100 steps of D = 20).

The scheme is not the reference's (OSHUN-1 has no implicit f00 step), so
these physics checks, not a reference run, pin it; the CUDA path is checked
against this restatement in tests/test_gpu_ee_implicit.py.
"""
import dataclasses

import numpy as np
import pytest

from oracle.cases import State, rel_l2
from tests.test_gpu_physics import _moments, _two_temperature_deck

SWEEPS = 3   # kEeImplicitSweeps of the CUDA path


def _run(oracle, d0, st0, D, sweeps, steps=1, small_dt=None):
    d = dataclasses.replace(d0, dt=D, small_dt=small_dt if small_dt else d0.small_dt)
    st = State(d, st0.f.copy(), st0.fields.copy())
    oracle.set_ee_implicit(sweeps)
    try:
        out = oracle.steps(st, steps, 2)
    finally:
        oracle.set_ee_implicit(0)
    return out.f[0, 0, 0].real


def _kurtosis(d, f00):
    p = d.pr()
    m0 = np.trapezoid(f00 * p ** 2, p)
    m2 = np.trapezoid(f00 * p ** 4, p)
    m4 = np.trapezoid(f00 * p ** 6, p)
    return m4 * m0 / m2 ** 2 - 5.0 / 3.0


def test_implicit_ee_converges_to_explicit(oracle):
    d0, st0 = _two_temperature_deck()
    f0 = st0.f[0, 0, 0].real
    diffs = []
    for D in (0.04, 0.02, 0.01):
        ex = _run(oracle, d0, st0, D, 0, small_dt=D / 20)
        be = _run(oracle, d0, st0, D, SWEEPS)
        diffs.append(rel_l2(be, ex))
        change = rel_l2(ex, f0)
        assert diffs[-1] <= 0.05 * change, (D, diffs[-1], change)
    assert diffs[0] / diffs[1] > 3.3 and diffs[1] / diffs[2] > 3.3, diffs


def test_implicit_ee_moments_follow_explicit(oracle):
    d0, st0 = _two_temperature_deck()
    n0, e0 = _moments(d0, st0.f[0, 0, 0].real)
    ex = _run(oracle, d0, st0, 2.0, 0, steps=5)
    be = _run(oracle, d0, st0, 2.0, SWEEPS, steps=5)
    n_e, e_e = _moments(d0, ex)
    n_b, e_b = _moments(d0, be)
    # the explicit scheme's own drifts are ~1.5e-6 (number) and ~2.3e-7 (energy)
    assert abs(n_b - n_e) <= 0.1 * abs(n_e - n0) + 1e-12 * n0, ((n_b - n0) / n0, (n_e - n0) / n0)
    assert abs(e_b - e_e) <= 0.1 * abs(e_e - e0) + 1e-12 * e0, ((e_b - e0) / e0, (e_e - e0) / e0)


def test_implicit_ee_large_steps_stay_positive(oracle):
    d0, st0 = _two_temperature_deck()
    n0, _ = _moments(d0, st0.f[0, 0, 0].real)
    k0 = _kurtosis(d0, st0.f[0, 0, 0].real)
    ex = _run(oracle, d0, st0, 200.0, 0, steps=10)      # 4000 explicit substeps
    f = _run(oracle, d0, st0, 200.0, SWEEPS, steps=10)
    assert np.all(np.isfinite(f)) and f.min() > 0.0
    n, _ = _moments(d0, f)
    assert abs(n - n0) <= 1e-4 * n0
    # both relax the two-temperature kurtosis (0.87) to the truncated grid's
    # equilibrium (~0.16); 3 sweeps of a 400-substep step land within 5 %
    assert k0 > 0.5 and _kurtosis(d0, f) < 0.25 * k0 and _kurtosis(d0, ex) < 0.25 * k0
    assert rel_l2(f, ex) <= 0.05
    f20 = _run(oracle, d0, st0, 20.0, SWEEPS, steps=100)
    assert rel_l2(f20, ex) <= 2e-3


@pytest.mark.parametrize("sweeps", [0, SWEEPS])
def test_oracle_ee_setting_is_restored(oracle, sweeps):
    """set_ee_implicit is process state of the checker: the default explicit
    scheme is back after each use above."""
    d0, st0 = _two_temperature_deck()
    a = _run(oracle, d0, st0, 2.0, sweeps)
    b = oracle.steps(State(dataclasses.replace(d0, dt=2.0), st0.f.copy(), st0.fields.copy()), 1, 2).f[0, 0, 0].real
    if sweeps == 0:
        assert np.array_equal(a, b)
    else:
        assert not np.array_equal(a, b)
