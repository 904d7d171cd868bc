"""The benchmarked configurations at their own sizes against the oracle.

* 2D2V Weibel, 128 x 128 cells, lmax = mmax = 6, np = 96 (three-cell FP64
  stage tiles, 43 tiles per row with a two-cell tail tile), two full small
  steps (RK4 Vlasov-Maxwell, e-e substeps, implicit f_lm) through the
  captured step graph, FP64: relative L2 <= 1e-12 per harmonic and field
  (same norm floor as every FP64 parity test).
* The same two steps in the FP32/FP64 split form: the relative L2 error of
  every harmonic and field against the FP64 oracle, without a norm floor,
  held to the per-result bounds below (f_22 and B_z carry the 1e-6 seed).
* A 128 x 8 strip of the same deck for 20 steps in the split form, every
  harmonic and field held to its own bound (twice the value measured on a
  B200): the m = 0 harmonics l = 1, 3, 4, 5, 6 carry small residuals of
  large E-field and advection terms and grow to 1e-6 .. 2e-5 there (their
  FP64 errors are 1e-11, against 1e-14 for the others, from the same
  sensitivity); everything else stays below 5e-7.
* 1D Landau damping, 64 cells, lmax = 8, np = 64, the full 1000 RK4 steps
  (dt = 0.05), FP64, <= 1e-12.

Reference sequence: Runge_Kutta_4::advance_p1 (OSHUN-1/def-RK.cpp:110-145),
Explicit_EC_FP::loop (def-FokkerPlanck.cpp:590-625), Euler_Backward
(def-FokkerPlanck.cpp:1270-1304).
"""
import numpy as np
import pytest

from oracle.cases import Deck, State, rel_l2
from oshun_b200 import workloads
from tests.gpu_util import run_gpu, worst_rel

pytestmark = pytest.mark.gpu
TOL = 1e-12

# FP32/FP64 split after two Weibel steps: unfloored relative L2 per result
# against the FP64 oracle.  Measured on a B200 (largest value over the
# harmonics of each group shown beside the bound).
FP32_BOUND_F00 = 1e-14          # f00 stays FP64 end to end
FP32_BOUND = 1e-6               # every other harmonic and field


def deck_of(cfg: dict) -> Deck:
    keys = ("l0", "m0", "nump", "numx", "numy", "NB_algorithms", "if_tridiagonal", "if_implicit1D", "pmin",
            "pmax", "xmin", "xmax", "ymin", "ymax", "dt", "small_dt", "density_np", "Zeta")
    return Deck(**{k: cfg[k] for k in keys})


def per_result(a: State, b: State):
    """Unfloored relative L2 error of every harmonic and field."""
    rows = {}
    for (l, m) in b.deck.harmonics():
        rows[f"f{l}{m}"] = rel_l2(a.harmonic(l, m), b.harmonic(l, m))
    for i, nm in enumerate(("Ex", "Ey", "Ez", "Bx", "By", "Bz")):
        rows[nm] = rel_l2(a.fields[i], b.fields[i])
    return rows


@pytest.fixture(scope="module")
def weibel_full(oracle):
    cfg, f, fields, _ = workloads.weibel2d(0)
    st = State(deck_of(cfg), f, fields)
    ref = oracle.steps(st, 2, 15)
    return st, ref


def test_weibel_full_size_fp64(weibel_full):
    st, ref = weibel_full
    out = run_gpu(st, ["step:2:15"], fast_path=True)
    err, where = worst_rel(out, ref)
    assert err <= TOL, (err, where)


def test_weibel_full_size_fp32_split_per_result(weibel_full):
    st, ref = weibel_full
    out = run_gpu(st, ["step:2:15"], fast_path=True, precision=1)
    rows = per_result(out, ref)
    assert rows["f00"] <= FP32_BOUND_F00, rows["f00"]
    bad = {k: v for k, v in rows.items() if k != "f00" and not v <= FP32_BOUND}
    assert not bad, bad


def test_landau_full_1000_steps(oracle):
    """Over 1000 steps the l = 7, 8 harmonics move by 2.5e-12 when f00 moves
    by one ulp, and the C restatement itself differs from the reference's
    own build by 2.3e-12 on l = 8 (measured on the CPU; the reference takes
    ~9 minutes for this run): every harmonic is held to 1e-12 or, where the
    problem's own rounding sensitivity is larger, to twice that sensitivity."""
    cfg, f, fields, _ = workloads.landau1d(0)
    st = State(deck_of(cfg), f, fields)
    ref = oracle.steps(st, 1000, 1)
    bumped = st.copy()
    bumped.f[0] *= 1.0 + 2.0 ** -52
    sens = oracle.steps(bumped, 1000, 1)
    out = run_gpu(st, ["step:1000:1"], fast_path=True)
    top = max(float(np.linalg.norm(ref.harmonic(l, m))) for (l, m) in st.deck.harmonics())
    for (l, m) in st.deck.harmonics():
        den = max(float(np.linalg.norm(ref.harmonic(l, m))), 1e-9 * top)
        s = float(np.linalg.norm(sens.harmonic(l, m) - ref.harmonic(l, m))) / den
        e = float(np.linalg.norm(out.harmonic(l, m) - ref.harmonic(l, m))) / den
        assert e <= max(TOL, 2.0 * s), ((l, m), e, s)
    nE = float(np.linalg.norm(ref.fields[0]))
    sE = float(np.linalg.norm(sens.fields[0] - ref.fields[0])) / nE
    eE = float(np.linalg.norm(out.fields[0] - ref.fields[0])) / nE
    assert eE <= max(TOL, 2.0 * sE), (eE, sE)
    # the damped field is still resolved: E_x carries the wave after 1000 steps
    assert np.linalg.norm(ref.fields[0]) > 0


# FP32/FP64 split, 128 x 8 strip, 20 steps: twice the measured relative L2
# error of each result against the FP64 oracle (unfloored)
STRIP_BOUNDS = {"f00": 1e-13, "f10": 2.5e-5, "f30": 4e-5, "f40": 8e-6, "f50": 3e-6, "f60": 1.3e-6,
                "f20": 2e-9}
STRIP_DEFAULT = 1e-6


def test_weibel_strip_fp32_split_20_steps(oracle):
    cfg, f, fields, _ = workloads.weibel2d(0, ny=8)
    st = State(deck_of(cfg), f, fields)
    ref = oracle.steps(st, 20, 15)
    out = run_gpu(st, ["step:20:15"], fast_path=True, precision=1)
    rows = per_result(out, ref)
    bad = {k: v for k, v in rows.items() if not v <= STRIP_BOUNDS.get(k, STRIP_DEFAULT)}
    assert not bad, bad
