"""The implicit electric field path (oshun_rk2_imp_step) against the
reference's own Runge_Kutta_2_Imp and Implicit_E_Field (the checker build's
istep op, OSHUN-1/main.cpp:77-107 with implicit_E; def-RK.cpp:399-588;
def-ImplicitE.cpp:471-676).

The RK2 actions alone (advance_p1: advection + B + Faraday; advance_p2: the
E couplings + CLEAN_LOW_PC) hold the FP64 bar of 1e-12.  The implicit E
itself comes from finite differences of the plasma's current under probe
fields of relative size sqrt(16 eps) = 6e-8, which amplify any rounding
difference by ~1e8: the reference's own output moves by ~3e-8 when every
element of its input moves by one ulp.  The full step is held to a small
multiple of that sensitivity, measured in the test on the same deck.
"""
import numpy as np
import pytest

from oracle.cases import Deck, State, run_reference, seeded_state
from tests.gpu_util import cfg_of, worst_rel

pytestmark = pytest.mark.gpu
TOL = 1e-12
SENS_FACTOR = 10.0    # full step: within this many times the reference's 1-ulp sensitivity


def _deck(one_d=False, **kw):
    base = dict(l0=4, m0=2, nump=24, numx=6, numy=1 if one_d else 4, xmax=2.0, ymax=3.0,
                if_implicit1D=1 if one_d else 0, dt=0.2, small_dt=0.1, density_np=1e25)
    base.update(kw)
    return Deck(**base)


def _state(d, seed):
    st = seeded_state(d, seed=seed, fields=d.numy > 1)
    if d.numy == 1:
        for (l, m) in d.harmonics():
            if m > 0:
                st.f[d.ind(l, m)] = 0
        st.fields[1:] = 0
        st.fields[0] = 1e-3 * np.cos(2 * np.pi * np.arange(d.numx) / d.numx)[None, :]
    return st


def run_imp(st, nsteps, mask):
    from oshun_b200 import Handle
    with Handle(**cfg_of(st.deck)) as h:
        h.upload(st.f, st.fields)
        h.rk2_imp_step(nsteps, mask)
        f, fl = h.download()
    return State(st.deck, f, fl)


@pytest.mark.parametrize("mask", [1, 32, 1 | 32, 1 | 2 | 32 | 4 | 8])
@pytest.mark.parametrize("one_d", [False, True])
def test_rk2_actions_match_reference(mask, one_d):
    d = _deck(one_d)
    st = _state(d, 71)
    ref = run_reference(st, [f"istep:1:{mask}"])
    err, where = worst_rel(run_imp(st, 1, mask), ref)
    assert err <= TOL, (err, where)


def ulp_noise(st, seed):
    """the state with every element moved by one ulp, up or down at random"""
    rng = np.random.default_rng(seed)
    out = st.copy()
    out.f = out.f * (1.0 + 2.0 ** -52 * rng.choice([-1.0, 1.0], size=out.f.shape))
    return out


@pytest.mark.parametrize("one_d", [False, True])
def test_implicit_step_within_reference_sensitivity(one_d):
    d = _deck(one_d)
    st = _state(d, 72)
    ref = run_reference(st, ["istep:1:63"])
    # the reference's own response to rounding-level changes of its input
    sens = max(worst_rel(run_reference(ulp_noise(st, k), ["istep:1:63"]), ref)[0] for k in (1, 2))
    err, where = worst_rel(run_imp(st, 1, 63), ref)
    print(f"implicit step ({'1D' if one_d else '2D'}): error {err:.3e} at {where}, reference sensitivity {sens:.3e}")
    assert err <= max(SENS_FACTOR * sens, TOL), (err, where, sens)
