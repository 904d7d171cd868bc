"""Collisional relaxation with heat flow (lmax = 1) at the configuration's
full size: nx = 256 periodic, np = 128 to 10 v_th, T(x) = T0 (1 + 1e-3 sin
kx), k lambda_ei over {0.01, 0.1, 1}.

* At dt = 0.1/nu_ei the explicit RK4 Vlasov-Maxwell step is unstable (w_p dt
  ~ 30) in the reference as here, so that dt runs the collision steps (f00
  e-e, implicit f1) alone, from a seeded f1;
* full steps (RK4 Vlasov-Maxwell + collisions) run at w_p dt = 0.5, where
  the temperature gradient drives the heat flux through advection.

FP64: relative L2 <= 1e-12 per harmonic and field against the oracle after 20
collision steps or 5 full steps (as for the Landau parity cases: at k
lambda_ei = 0.01 f1 is ~4e-7 of f00 and E_x ~3e-9, both made by cancelling
sums whose rounding differences grow with every step; after 10 steps they
reach 1.05e-12), number and energy drift equal to the oracle's; the
FP32/FP64-split form: <= 1e-6 against the same FP64 oracle (f00 and the
collision arithmetic stay FP64).
"""
import numpy as np
import pytest

from oracle.cases import Deck, State
from tests.gpu_util import worst_rel

pytestmark = pytest.mark.gpu
NSTEPS = 20         # collision steps
NSTEPS_FULL = 5     # full steps


def _deck(cfg) -> Deck:
    return Deck(l0=cfg["l0"], m0=cfg["m0"], nump=cfg["nump"], numx=cfg["numx"], numy=1,
                NB_algorithms=cfg["NB_algorithms"], if_tridiagonal=cfg["if_tridiagonal"],
                if_implicit1D=cfg["if_implicit1D"], pmin=cfg["pmin"], pmax=cfg["pmax"], xmin=cfg["xmin"],
                xmax=cfg["xmax"], dt=cfg["dt"], small_dt=cfg["small_dt"], density_np=cfg["density_np"],
                Zeta=cfg["Zeta"])


def _moments(p, f00):
    n = np.sum(np.trapezoid(f00.real * p ** 2, p, axis=-1))
    e = np.sum(np.trapezoid(f00.real * p ** 2 * (np.sqrt(1 + p * p) - 1), p, axis=-1))
    return n, e


def _case(klam, full):
    from oshun_b200 import workloads
    cfg, f, fields, meta = workloads.relax1d(klam_ei=klam, dt=0.5 if full else None)
    st = State(_deck(cfg), f, fields)
    if not full:
        # a heat-flux-like f1 for the implicit f1 solve to relax
        p = st.deck.pr()
        x = np.arange(st.deck.numx) * (2 * np.pi / st.deck.numx)
        st.f[1, 0] = 1e-3 * np.sin(x)[:, None] * p[None, :] * st.f[0, 0].real
    return cfg, st, (15 if full else 14), (NSTEPS_FULL if full else NSTEPS)


def _run(cfg, st, mask, nsteps, precision):
    from oshun_b200 import Handle
    c = dict(cfg)
    c["precision"] = precision
    with Handle(**c) as h:
        h.upload(st.f, st.fields)
        if mask == 15:
            h.step(nsteps, collisions=True)
        else:
            t = 0.0
            for _ in range(nsteps):
                t += st.deck.dt
                h.collide_ee(t)
                h.collide_f1(t)
                h.collide_flm(t)
        f, fl = h.download()
    return State(st.deck, f, fl)


# k lambda_ei changes only the cell size, so the collision-only case runs once
@pytest.mark.parametrize("klam,full", [(0.1, False), (0.01, True), (0.1, True), (1.0, True)])
def test_relax_fp64_parity(oracle, klam, full):
    cfg, st, mask, nsteps = _case(klam, full)
    ref = oracle.steps(st, nsteps, mask)
    got = _run(cfg, st, mask, nsteps, 0)
    err, where = worst_rel(got, ref)
    assert err <= 1e-12, (err, where)
    p = st.deck.pr()
    n0, e0 = _moments(p, st.f[0, 0])
    ng, eg = _moments(p, got.f[0, 0])
    nr, er = _moments(p, ref.f[0, 0])
    assert abs(ng - nr) <= 1e-13 * n0 and abs(eg - er) <= 1e-12 * e0
    assert abs(ng - n0) <= 1e-5 * n0 and abs(eg - e0) <= 1e-3 * e0


@pytest.mark.parametrize("full", [False, True])
def test_relax_fp32_split(oracle, full):
    cfg, st, mask, nsteps = _case(0.1, full)
    ref = oracle.steps(st, nsteps, mask)
    got = _run(cfg, st, mask, nsteps, 1)
    err, where = worst_rel(got, ref, floor=1e-3)
    assert err <= 1e-6, (err, where)
