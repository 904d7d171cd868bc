"""The FP32/FP64-split form (OSHUN_FP32_SPLIT) against the FP64 checker.

l >= 1 harmonics, fields and the RHS arithmetic in FP32; f00, the current
reduction, the e-e step, the Rosenbluth integrals and the collision
coefficients and solves in FP64.  Error is stated per harmonic: relative L2
against the FP64 restatement, bar 1e-6 for harmonics carrying at least 1e-3 of
the largest harmonic's norm (smaller ones are held to the same absolute error
as that floor: FP32 resolves a harmonic only relative to what feeds it).
"""
import numpy as np
import pytest

from oracle.cases import Deck, seeded_state
from tests.gpu_util import run_gpu, worst_rel

pytestmark = pytest.mark.gpu
TOL = 1e-6


@pytest.mark.parametrize("kw,ops,mask", [
    (dict(l0=6, m0=6, nump=32, numx=6, numy=6, if_implicit1D=0, dt=0.02, small_dt=0.05, density_np=1e21), "rhs", None),
    (dict(l0=6, m0=6, nump=32, numx=6, numy=6, if_implicit1D=0, dt=0.02, small_dt=0.05, density_np=1e21), "step:5:15", 15),
    (dict(l0=8, m0=0, nump=64, numx=16, numy=1, if_implicit1D=1, dt=0.05, small_dt=0.05, density_np=1e21), "step:10:15", 15),
])
def test_fp32_split_error(oracle, kw, ops, mask):
    d = Deck(xmax=2.0, ymax=3.0, **kw)
    st = seeded_state(d, seed=41, fields=d.numy > 1)
    if d.numy == 1:
        for (l, m) in d.harmonics():
            if m > 0:
                st.f[d.ind(l, m)] = 0
        st.fields[1:] = 0
    got = run_gpu(st, [ops], precision=1)
    ref = oracle.rhs(st) if ops == "rhs" else oracle.steps(st, int(ops.split(":")[1]), mask)
    err, where = worst_rel(got, ref, floor=1e-3)
    assert err <= TOL, (err, where)
    # and the FP64 drop-in is far closer
    if ops != "rhs":
        err64, _ = worst_rel(run_gpu(st, [ops]), ref)
        assert err64 <= 1e-12


def test_fp32_split_keeps_f00_fp64(oracle):
    """f00 stays FP64: a collisions-only step (e-e plus implicit f_lm) of the
    split form matches the FP64 checker on f00 at FP64 accuracy."""
    d = Deck(l0=3, m0=0, nump=64, numx=4, numy=1, if_implicit1D=1, dt=0.4, small_dt=0.15, density_np=5e24,
             xmax=2.0)
    st = seeded_state(d, seed=42, fields=False)
    got = run_gpu(st, ["step:2:2"], precision=1)
    ref = oracle.steps(st, 2, 2)
    a, b = got.harmonic(0, 0), ref.harmonic(0, 0)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-12
