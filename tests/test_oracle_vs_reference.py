"""The C restatement against the reference's own code on fresh seeded inputs
(needs oracle/_ref/oshun_ref, built from the reference sources)."""
import pytest

from oracle.cases import Deck, reference_available, run_reference, seeded_state
from tests.gpu_util import worst_rel

pytestmark = pytest.mark.skipif(not reference_available(), reason="reference checker not built")
TOL = 1e-12


def _zero_m(st):
    for (l, m) in st.deck.harmonics():
        if m > 0:
            st.f[st.deck.ind(l, m)] = 0
    st.fields[1:] = 0
    return st


CASES = [
    # (deck kwargs, ops, seed)
    (dict(l0=5, m0=2, nump=20, numx=8, numy=1, if_implicit1D=1, dt=0.4, small_dt=0.15, density_np=3e24), ["rhs"], 1),
    (dict(l0=5, m0=2, nump=20, numx=8, numy=1, if_implicit1D=1, dt=0.4, small_dt=0.15, density_np=3e24), ["step:2:15"], 2),
    (dict(l0=4, m0=4, nump=12, numx=4, numy=6, if_implicit1D=0, dt=0.2, small_dt=0.1, density_np=1e25), ["rhs"], 3),
    (dict(l0=7, m0=3, nump=12, numx=5, numy=4, if_implicit1D=0, dt=0.2, small_dt=0.1, density_np=1e25), ["rhs"], 4),
    (dict(l0=5, m0=3, nump=12, numx=4, numy=4, if_implicit1D=0, dt=0.2, small_dt=0.1, density_np=1e25), ["step:2:15"], 5),
    (dict(l0=4, m0=2, nump=12, numx=4, numy=4, if_implicit1D=0, if_tridiagonal=0, dt=0.2, small_dt=0.07,
          density_np=1e25), ["step:2:15"], 6),
    (dict(l0=3, m0=2, nump=24, numx=4, numy=1, if_implicit1D=1, if_tridiagonal=0, dt=1.0, small_dt=0.3,
          density_np=1e26, NB_algorithms=6), ["step:2:14"], 7),
]


@pytest.mark.parametrize("kw,ops,seed", CASES)
def test_oracle_vs_reference(oracle, kw, ops, seed):
    d = Deck(xmax=2.0, ymax=3.0, **kw)
    st = seeded_state(d, seed=seed, fields=d.numy > 1)
    if d.numy == 1:
        st = _zero_m(st)
    ref = run_reference(st, ops)
    out = st
    for op in ops:
        if op == "rhs":
            out = oracle.rhs(out)
        else:
            p = op.split(":")
            out = oracle.steps(out, int(p[1]), int(p[2]))
    err, where = worst_rel(out, ref)
    assert err <= TOL, (err, where)


def test_reference_yadv_chain_factor_is_real(oracle):
    """Dropping the reference's y-advection chain factor (m >= 2) breaks
    parity: the factor is part of the reference's behaviour."""
    d = Deck(l0=6, m0=6, nump=10, numx=4, numy=4, xmax=2.0, ymax=3.0, if_implicit1D=0)
    st = seeded_state(d, seed=9)
    ref = run_reference(st, ["rhs"])
    oracle.set_yadv_chain(False)
    try:
        err, _ = worst_rel(oracle.rhs(st), ref)
    finally:
        oracle.set_yadv_chain(True)
    assert err > 1e-3


def nondominant_case():
    """A dense-mode deck whose l = 3 matrices fail the reference's dominance
    test in every cell (f00 negated, so the scattering term turns the diagonal
    negative): Gauss_Seidel returns false and the solve keeps f
    (OSHUN-1/def-Nmethods.cpp:70-76, def-FokkerPlanck.cpp:1021-1032)."""
    d = Deck(l0=3, m0=2, nump=24, numx=4, numy=1, if_implicit1D=1, if_tridiagonal=0, dt=5.0, small_dt=5.0,
             density_np=1e21, xmax=2.0)
    st = _zero_m(seeded_state(d, seed=5, fields=False))
    st.f[0] *= -1.0
    return st


def test_nondominant_skip_matches_reference(oracle):
    import numpy as np
    st = nondominant_case()
    d = st.deck
    ref = run_reference(st, ["step:1:12"])
    out = oracle.steps(st, 1, 12)
    assert oracle.nondominant() == d.numx          # one skipped solve (l = 3) per cell
    err, where = worst_rel(out, ref)
    assert err <= TOL, (err, where)
    assert np.array_equal(ref.harmonic(3, 0), st.harmonic(3, 0))      # kept
    assert not np.array_equal(ref.harmonic(2, 0), st.harmonic(2, 0))  # solved
