"""Physics checks of the CUDA path at full configuration sizes.

* Landau damping (1D, k lambda_D = 0.3, lmax = 8, 64 cells, np = 64 to 8 v_th,
  RK4 dt = 0.05/w_p, 1000 steps): the fitted damping rate of the field energy
  against the analytic rate.  The analytic rate is the root of the kinetic
  dispersion relation 1 + (1 + zeta Z(zeta))/(k lambda_D)^2 = 0 (computed here
  with the Faddeeva function), corrected for the relativistic Maxwellian at
  v_th = 0.05 c by the ratio of the weak-damping rates
  -eps_i/(d eps_r/d omega) of the relativistic (Gaussian in p, v = p/gamma)
  and the non-relativistic distribution (computed here by quadrature).
* e-e collisions: number and energy drift of the GPU equal the reference
  scheme's drift (the C restatement) and stay small; a two-temperature f00
  relaxes toward a Maxwellian.
"""
import numpy as np
import pytest

from oracle.cases import Deck, State, maxwellian, rel_l2
from tests.gpu_util import cfg_of

pytestmark = pytest.mark.gpu


# ---------------------------------------------------------------------------
# analytic Landau rate
# ---------------------------------------------------------------------------

def _nonrel_root(klam):
    from scipy.special import wofz

    def eps(w):
        zeta = w / (np.sqrt(2.0) * klam)
        return 1.0 + (1.0 + zeta * 1j * np.sqrt(np.pi) * wofz(zeta)) / klam ** 2
    w = 1.16 - 0.01j
    for _ in range(60):
        h = 1e-7
        w = w - eps(w) / ((eps(w + h) - eps(w - h)) / (2 * h))
    return w


def _weak_damping_rate(vth, klam, relativistic):
    """-eps_i/(d eps_r/d omega) at the real root, for the Gaussian-in-p
    Maxwellian with v = p/gamma (relativistic) or v = p."""
    from scipy import integrate, optimize
    k = klam / vth

    def f0(px, pp):
        return np.exp(-(px * px + pp * pp) / (2 * vth * vth)) / ((2 * np.pi) ** 1.5 * vth ** 3)

    def v_of(px, pp):
        return px / np.sqrt(1 + px * px + pp * pp) if relativistic else px

    def eps_r(w):
        u = w / k

        def inner(pp):
            s = np.sqrt(1 + pp * pp) if relativistic else 1.0
            vmax = 12 * vth / np.sqrt(1 + 144 * vth * vth) if relativistic else 12 * vth

            def g(v):
                if relativistic:
                    px = v * s / np.sqrt(1 - v * v)
                    jac = s / (1 - v * v) ** 1.5
                else:
                    px, jac = v, 1.0
                return -px / vth ** 2 * f0(px, pp) * jac / k
            val, _ = integrate.quad(g, -vmax, vmax, weight="cauchy", wvar=u, limit=400)
            return 2 * np.pi * pp * val
        tot, _ = integrate.quad(inner, 0, 10 * vth, limit=200)
        return 1 - tot / k

    def eps_i(w):
        u = w / k

        def inner(pp):
            if relativistic:
                s = np.sqrt(1 + pp * pp)
                px = u * s / np.sqrt(1 - u * u)
                gam = np.sqrt(1 + px * px + pp * pp)
                dvdp = (1 + pp * pp) / gam ** 3
            else:
                px, dvdp = u, 1.0
            return 2 * np.pi * pp * (-px / vth ** 2 * f0(px, pp)) / (k * dvdp)
        tot, _ = integrate.quad(inner, 0, 10 * vth, limit=200)
        return -(np.pi / k) * tot

    wr = optimize.brentq(eps_r, 1.0, 1.5)
    h = 1e-5
    return -eps_i(wr) / ((eps_r(wr + h) - eps_r(wr - h)) / (2 * h))


def analytic_landau_rate(vth, klam=0.3):
    exact = _nonrel_root(klam).imag
    ratio = _weak_damping_rate(vth, klam, True) / _weak_damping_rate(vth, klam, False)
    return exact * ratio


def fitted_rate(W, dt, t_lo=3.0, t_hi=40.0):
    t = dt * np.arange(1, len(W) + 1)
    pk = [i for i in range(1, len(W) - 1) if W[i] > W[i - 1] and W[i] >= W[i + 1]]
    tp, wp = t[pk], W[pk]
    sel = (tp > t_lo) & (tp < t_hi)
    assert sel.sum() >= 8
    return np.polyfit(tp[sel], np.log(wp[sel]), 1)[0] / 2.0


@pytest.mark.parametrize("vth", [0.05, 0.01])
def test_landau_damping_rate(vth):
    from oshun_b200 import Handle, workloads
    cfg, f, fields, meta = workloads.landau1d(vth=vth)
    W = []
    with Handle(**cfg) as h:
        h.upload(f, fields)
        for _ in range(1000):
            h.step(1, collisions=False)
            _, fl = h.download()
            W.append(float(np.sum(fl[0].real ** 2)))
    gamma = fitted_rate(np.array(W), cfg["dt"])
    expect = analytic_landau_rate(vth)
    assert abs(gamma - expect) <= 0.05 * abs(expect), (gamma, expect)


def test_landau_charge_conservation(oracle):
    """Total electron number (trapezoid in p of f00 p^2, summed over x) over
    200 collisionless steps: the GPU's drift equals the reference scheme's
    (the C restatement) and is small."""
    from oracle.cases import Deck, State
    from oshun_b200 import Handle, workloads
    cfg, f, fields, meta = workloads.landau1d()
    p = workloads.p_axis(cfg["nump"], cfg["pmin"], cfg["pmax"])

    def number(f00):
        return float(np.sum(np.trapezoid(f00.real * p ** 2, p, axis=-1)))
    n0 = number(f[0, 0])
    with Handle(**cfg) as h:
        h.upload(f, fields)
        h.step(200, collisions=False)
        f1, _ = h.download()
    d = Deck(l0=cfg["l0"], m0=0, nump=cfg["nump"], numx=cfg["numx"], numy=1, pmin=cfg["pmin"], pmax=cfg["pmax"],
             xmin=cfg["xmin"], xmax=cfg["xmax"], dt=cfg["dt"])
    ref = oracle.steps(State(d, f, fields), 200, 1)
    n_gpu, n_ref = number(f1[0, 0]), number(ref.f[0, 0])
    assert abs(n_gpu - n_ref) <= 1e-12 * n0
    assert abs(n_gpu - n0) <= 1e-6 * n0


# ---------------------------------------------------------------------------
# e-e collisions: conservation and relaxation
# ---------------------------------------------------------------------------

def _two_temperature_deck():
    d = Deck(l0=2, m0=0, nump=96, numx=4, numy=1, pmax=0.4, dt=2.0, small_dt=0.5, density_np=1e24,
             if_implicit1D=1, xmax=1.0)
    st = State(d)
    p = d.pr()
    f = 0.7 * maxwellian(p, 0.04) + 0.3 * maxwellian(p, 0.08)
    st.f[0, 0, :, :] = f[None, :]
    return d, st


def _moments(d, f00):
    p = d.pr()
    v = p / np.sqrt(1 + p * p)
    dv = np.diff(v)
    n = np.sum(0.5 * (v[1:] ** 2 * f00[1:] + v[:-1] ** 2 * f00[:-1]) * dv)
    e = np.sum(0.5 * (v[1:] ** 4 * f00[1:] + v[:-1] ** 4 * f00[:-1]) * dv)
    return n, e


def test_ee_conservation_matches_reference_scheme(oracle):
    from oshun_b200 import Handle
    d, st = _two_temperature_deck()
    n0, e0 = _moments(d, st.f[0, 0, 0].real)
    ref = oracle.steps(st, 5, 2)
    with Handle(**cfg_of(d)) as h:
        h.upload(st.f, st.fields)
        t = 0.0
        for _ in range(5):
            t += d.dt
            h.collide_ee(t)
        f, _ = h.download()
    n_g, e_g = _moments(d, f[0, 0, 0].real)
    n_r, e_r = _moments(d, ref.f[0, 0, 0].real)
    assert abs(n_g - n_r) <= 1e-12 * n0 and abs(e_g - e_r) <= 1e-12 * e0
    assert abs(n_g - n0) <= 1e-5 * n0 and abs(e_g - e0) <= 1e-5 * e0
    assert rel_l2(f[0, 0, 0].real, ref.f[0, 0, 0].real) <= 1e-12


def test_ee_relaxes_toward_maxwellian():
    """The kurtosis of the two-temperature distribution moves toward the
    Maxwellian value under e-e collisions."""
    from oshun_b200 import Handle
    d, st = _two_temperature_deck()
    p = d.pr()

    def excess_kurtosis(f00):
        m2 = np.trapezoid(f00 * p ** 4, p)
        m0 = np.trapezoid(f00 * p ** 2, p)
        m4 = np.trapezoid(f00 * p ** 6, p)
        return m4 * m0 / m2 ** 2 - 5.0 / 3.0     # 3D isotropic Maxwellian: <p^4><1>/<p^2>^2 = 5/3
    k = [excess_kurtosis(st.f[0, 0, 0].real)]
    with Handle(**cfg_of(d)) as h:
        h.upload(st.f, st.fields)
        t = 0.0
        for _ in range(6):
            t += 20 * d.dt
            h.collide_ee(t)
            f, _ = h.download()
            k.append(excess_kurtosis(f[0, 0, 0].real))
    assert k[0] > 0.05
    assert all(b < a for a, b in zip(k, k[1:]))
    assert k[-1] < 0.9 * k[0]
