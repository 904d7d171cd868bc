"""Failure paths of the CUDA path, each made safely (no GPU fault, trap or
hang; every device wait is bounded):

* a NaN in the uploaded state: the status word's bit 1 after the step;
* a dense-mode matrix that fails the reference's diagonal-dominance test:
  bit 0, the skip count, and the skipped planes kept as the reference keeps
  them (OSHUN-1/def-Nmethods.cpp:70-76, def-FokkerPlanck.cpp:1021-1032);
* a stage-kernel pipeline wait that runs out (a copy withheld by the test
  hook, waits shortened to 2 ms): the launch returns, bit 4 is set, and the
  handle's next step is exact again.
"""
import numpy as np
import pytest

from oracle.cases import Deck, seeded_state
from tests.gpu_util import cfg_of, run_gpu, worst_rel
from tests.test_oracle_vs_reference import nondominant_case

pytestmark = pytest.mark.gpu


def _deck():
    return Deck(l0=4, m0=2, nump=32, numx=6, numy=4, if_implicit1D=0, if_tridiagonal=1, dt=0.2, small_dt=0.07,
                density_np=1e25, xmax=2.0, ymax=3.0)


def test_nan_in_state_sets_numeric_bit(oracle):
    from oshun_b200 import Handle
    d = _deck()
    st = seeded_state(d, seed=31)
    bad = st.copy()
    bad.f[d.ind(0, 0), 1, 2, 5] = np.nan
    with Handle(**cfg_of(d)) as h:
        h.upload(bad.f, bad.fields)
        h.step(1, collisions=True)
        flags, _ = h.status_flags()
        assert flags & 2, flags
        # the word clears on reading, and a clean state steps exactly again
        h.upload(st.f, st.fields)
        h.step(1, collisions=True)
        flags, _ = h.status_flags()
        assert flags == 0, flags
        f, fl = h.download()
    from oracle.cases import State
    err, where = worst_rel(State(d, f, fl), oracle.steps(st, 1, 15))
    assert err <= 1e-12, (err, where)


def test_nondominant_solve_is_skipped_and_counted(oracle):
    from oshun_b200 import Handle
    st = nondominant_case()
    d = st.deck
    ref = oracle.steps(st, 1, 12)
    want = oracle.nondominant()
    with Handle(**cfg_of(d)) as h:
        h.upload(st.f, st.fields)
        h.collide_f1(d.dt)
        h.collide_flm(d.dt)
        flags, count = h.status_flags()
        f, fl = h.download()
    assert flags & 1, flags
    assert count == want == d.numx, (count, want)
    from oracle.cases import State
    out = State(d, f, fl)
    assert np.array_equal(out.harmonic(3, 0), st.harmonic(3, 0))   # kept, bit for bit
    err, where = worst_rel(out, ref)
    assert err <= 1e-12, (err, where)


@pytest.mark.parametrize("withhold", [0, 7])
def test_stage_wait_timeout_returns_and_recovers(oracle, withhold):
    from oshun_b200 import Handle
    from oracle.cases import State
    d = _deck()
    st = seeded_state(d, seed=32)
    with Handle(**cfg_of(d)) as h:
        h.upload(st.f, st.fields)
        h.inject_stage_timeout(withhold, 2e-3)
        h.rk4_step()
        h.synchronize()
        flags, _ = h.status_flags()
        assert flags & 16, flags
        # the handle is usable: re-upload and step exactly
        h.upload(st.f, st.fields)
        h.rk4_step()
        h.synchronize()
        flags, _ = h.status_flags()
        assert flags == 0, flags
        f, fl = h.download()
    err, where = worst_rel(State(d, f, fl), oracle.steps(st, 1, 1))
    assert err <= 1e-12, (err, where)
