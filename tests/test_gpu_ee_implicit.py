"""The opt-in backward-Euler f00 e-e step (OSHUN_FLAG_IMPLICIT_EE) on the
GPU against its C restatement in the oracle (the scheme is not the
reference's; tests/test_ee_implicit_oracle.py pins the restatement to the
reference's explicit scheme by convergence, conservation and stability):

* the two-temperature relaxation deck, 5 steps of D = 2 and 10 steps of
  D = 200 through oshun_collide_ee: relative L2 <= 1e-12;
* full steps (RK4 + implicit e-e + implicit f_lm) through the captured step
  graph on a 2D deck, tridiagonal and dense: <= 1e-12 per harmonic and field;
* batches refuse the flag (their collision groups run the explicit substeps).
"""
import dataclasses

import numpy as np
import pytest

from oracle.cases import Deck, State, rel_l2, seeded_state
from tests.gpu_util import cfg_of, run_gpu, worst_rel
from tests.test_gpu_physics import _two_temperature_deck

pytestmark = pytest.mark.gpu
TOL = 1e-12
SWEEPS = 3
FLAG = 0x2   # OSHUN_FLAG_IMPLICIT_EE


def _oracle_steps(oracle, st, n, mask):
    oracle.set_ee_implicit(SWEEPS)
    try:
        return oracle.steps(st, n, mask)
    finally:
        oracle.set_ee_implicit(0)


@pytest.mark.parametrize("D,n", [(2.0, 5), (200.0, 10)])
def test_implicit_ee_matches_oracle(oracle, D, n):
    from oshun_b200 import Handle
    d0, st0 = _two_temperature_deck()
    d = dataclasses.replace(d0, dt=D)
    st = State(d, st0.f.copy(), st0.fields.copy())
    ref = _oracle_steps(oracle, st, n, 2)
    with Handle(**cfg_of(d, flags=FLAG)) as h:
        h.upload(st.f, st.fields)
        t = 0.0
        for _ in range(n):
            t += D
            h.collide_ee(t)
        f, _ = h.download()
    for c in range(d.numx):
        assert rel_l2(f[0, 0, c].real, ref.f[0, 0, c].real) <= TOL
    assert np.all(f[0, 0].real > 0)


@pytest.mark.parametrize("tri", [1, 0])
def test_implicit_ee_full_steps_match_oracle(oracle, tri):
    d = Deck(l0=4, m0=2, nump=32, numx=6, numy=4, if_implicit1D=0, if_tridiagonal=tri,
             dt=0.3, small_dt=0.07, density_np=1e25, xmax=2.0, ymax=3.0)
    st = seeded_state(d, seed=31)
    ref = _oracle_steps(oracle, st, 3, 15)
    out = run_gpu(st, ["step:3:15"], fast_path=True, flags=FLAG)
    err, where = worst_rel(out, ref)
    assert err <= TOL, (err, where)
    # and it is not the explicit scheme: the e-e step changed f00 differently
    exp = oracle.steps(st, 3, 15)
    assert rel_l2(out.f[0], exp.f[0]) > 1e-9


def test_batch_refuses_implicit_ee():
    from oshun_b200 import Batch, OshunError
    d, _ = _two_temperature_deck()
    with pytest.raises(OshunError):
        Batch([cfg_of(d, flags=FLAG)])
    Batch([cfg_of(d, flags=FLAG)], collide=[False]).close()
