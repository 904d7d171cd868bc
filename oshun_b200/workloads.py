"""Synthetic, seeded workloads of the benchmark configurations.

Every builder returns ``(cfg, f, fields, meta)``: ``cfg`` the oshun_cfg
fields, ``f`` complex128 [Nh][numy][numx][nump] and ``fields`` complex128
[6][numy][numx] in the reference's storage order (ind(l,m),
OSHUN-1/def-State.cpp:420-427), ``meta`` a description.  Units are the
reference's: p in m_e c, x in c/w_p, t in 1/w_p (OSHUN-1/def-Input.cpp:77-80).
The Maxwellian is the reference's Gaussian_p normalisation,
exp(-p^2/2pt^2)/((2 pi)^{3/2} pt^3) (OSHUN-1/def-Setup.cpp:500-533).
"""
from __future__ import annotations

import numpy as np

WORKLOADS = ("weibel2d", "weibel2d_64", "landau1d", "relax1d", "landau1d_large")


def num_harmonics(l0: int, m0: int) -> int:
    return ((m0 + 1) * (2 * l0 - m0 + 2)) // 2


def ind(l: int, m: int, m0: int) -> int:
    return (l * (l + 1)) // 2 + m if l < m0 + 1 else l * (m0 + 1) - (m0 * (m0 + 1)) // 2 + m


def p_axis(nump: int, pmin: float, pmax: float) -> np.ndarray:
    return np.arange(nump, dtype=np.float64) * ((pmax - pmin) / (nump - 1)) + pmin


def maxwellian(p, pt):
    return np.exp(-(p * p) / (2.0 * pt * pt)) / (np.sqrt(2.0 * np.pi) * 2.0 * np.pi * pt ** 3)


def _base_cfg(**kw) -> dict:
    cfg = dict(t0=0.0, NB_algorithms=4, if_tridiagonal=1, if_implicit1D=1, density_np=1e21, Zeta=1.0,
               ymin=0.0, ymax=1.0, precision=0, flags=0, small_dt=1.0)
    cfg.update(kw)
    return cfg


def weibel2d(precision: int = 0, seed: int = 7, nx: int = 128, ny: int = 128):
    """2D2V Weibel-type: nx = ny = 128 periodic, lmax = mmax = 6, np = 96 to
    p_max = 8 v_th, bi-Maxwellian T_x/T_y = 4 projected onto l = 0, 2 (m = 0)
    with seeded m = 2 noise, seeded B_z noise of amplitude 1e-6, full E and B
    update, anisotropic collisions (tridiagonal, the production setting of the
    reference's paper decks) at nu/w_p ~ 1e-3, RK4 dt = 0.02/w_p."""
    vth = 0.05
    l0 = m0 = 6
    nump = 96
    pmax = 8.0 * vth
    pmin = pmax / (2.0 * nump)
    L = 2.0 * np.pi / 0.5            # k_min = 0.5 w_p/c
    cfg = _base_cfg(l0=l0, m0=m0, nump=nump, numx=nx, numy=ny, pmin=pmin, pmax=pmax,
                    xmin=0.0, xmax=L * (nx - 1) / nx, ymin=0.0, ymax=L * (ny - 1) / ny,
                    dt=0.02, small_dt=0.05, if_implicit1D=0, if_tridiagonal=1,
                    density_np=1e21, precision=precision)
    rng = np.random.default_rng(seed)
    p = p_axis(nump, pmin, pmax)
    # bi-Maxwellian, anisotropy axis x (the polar axis of the harmonics)
    Tx, Ty = (2.0 * vth) ** 2, vth ** 2
    mu, w = np.polynomial.legendre.leggauss(64)
    P, MU = np.meshgrid(p, mu, indexing="ij")
    fb = np.exp(-(P * MU) ** 2 / (2 * Tx) - P ** 2 * (1 - MU ** 2) / (2 * Ty))
    fb /= (2 * np.pi) ** 1.5 * np.sqrt(Tx) * Ty
    f00 = 0.5 * (fb * w).sum(axis=1)
    P2 = 0.5 * (3 * mu ** 2 - 1)
    f20 = 2.5 * (fb * (w * P2)).sum(axis=1)
    nh = num_harmonics(l0, m0)
    f = np.zeros((nh, ny, nx, nump), np.complex128)
    f[ind(0, 0, m0)] = f00[None, None, :]
    f[ind(2, 0, m0)] = f20[None, None, :]
    noise = 1e-6 * rng.standard_normal((ny, nx)) + 1e-6j * rng.standard_normal((ny, nx))
    f[ind(2, 2, m0)] = noise[..., None] * f20[None, None, :]
    fields = np.zeros((6, ny, nx), np.complex128)
    fields[5] = 1e-6 * rng.standard_normal((ny, nx))
    meta = dict(workload="weibel2d", nx=nx, ny=ny, lmax=l0, mmax=m0, np=nump, vth=vth,
                anisotropy="Tx/Ty=4", collisions="ee + implicit flm, tridiagonal", dt=0.02)
    return cfg, f, fields, meta


def weibel2d_64(precision: int = 0):
    """The Weibel configuration on 64 x 64 cells (profiling size: 154 MB per
    FP64 state copy, still larger than L2)."""
    cfg, f, fields, meta = weibel2d(precision, nx=64, ny=64)
    meta["workload"] = "weibel2d_64"
    return cfg, f, fields, meta


def landau1d(precision: int = 0, nx: int = 64, nump: int = 64, l0: int = 8, alpha: float = 1e-3,
             klam: float = 0.3, vth: float = 0.05):
    """1D1P Landau damping: nx periodic cells over L = 2 pi/k with
    k lambda_D = klam, v_th = 0.05c, np cells to 8 v_th, n = 1 + alpha cos kx,
    E_x from Gauss's law, fixed neutralising ions, RK4 dt = 0.05/w_p."""
    k = klam / vth
    L = 2.0 * np.pi / k
    pmax = 8.0 * vth
    pmin = pmax / (2.0 * nump)
    cfg = _base_cfg(l0=l0, m0=0, nump=nump, numx=nx, numy=1, pmin=pmin, pmax=pmax, xmin=0.0,
                    xmax=L * (nx - 1) / nx, dt=0.05, precision=precision)
    p = p_axis(nump, pmin, pmax)
    x = np.arange(nx) * (L / nx)
    n = 1.0 + alpha * np.cos(k * x)
    f = np.zeros((num_harmonics(l0, 0), 1, nx, nump), np.complex128)
    f[0, 0] = n[:, None] * maxwellian(p[None, :], vth)
    fields = np.zeros((6, 1, nx), np.complex128)
    fields[0, 0] = -alpha / k * np.sin(k * x)
    meta = dict(workload="landau1d", nx=nx, np=nump, lmax=l0, klambdaD=klam, vth=vth, dt=0.05)
    return cfg, f, fields, meta


def landau1d_large(precision: int = 0):
    """Landau damping at nx = 8192, np = 256, lmax = 16: 35.7 M coefficients."""
    cfg, f, fields, meta = landau1d(precision, nx=8192, nump=256, l0=16)
    meta["workload"] = "landau1d_large"
    return cfg, f, fields, meta


def relax1d(precision: int = 0, klam_ei: float = 0.1, nx: int = 256, nump: int = 128, vth: float = 0.05,
            dt: float | None = None, ee_substeps: int = 10):
    """Collisional relaxation with heat flow: nx = 256 periodic, T(x) = T0
    (1 + 1e-3 sin kx), uniform density, Z = 1, lmax = 1, np = 128 to 10 v_th,
    implicit f1 solve and the f00 e-e step every step.

    dt defaults to 0.1/nu_ei.  The reference's f00 e-e step is explicit RK4
    subcycled at small_dt (Explicit_EC_FP::loop, def-FokkerPlanck.cpp:590-625);
    at dt = 0.1/nu_ei it needs ~10 substeps to stay stable, so small_dt =
    dt/ee_substeps.  The explicit RK4 Vlasov-Maxwell step is stable only for
    w_p dt and v dt/dx of order 1, far below 0.1/nu_ei: at that dt the
    configuration runs collision steps only."""
    pmax = 10.0 * vth
    pmin = pmax / (2.0 * nump)
    density = 1e22
    # electron-ion collision frequency at v_th from the reference's scattering
    # term: nu ~ Z lnL_ei * re * kp / v_th^3 (def-FokkerPlanck.cpp:785-787, 872-879)
    re = 2.8179402894e-13
    kp = np.sqrt(4.0 * np.pi * density * re)
    nu = 8.0 * re * kp / vth ** 3
    lam_ei = vth / nu
    k = klam_ei / lam_ei
    L = 2.0 * np.pi / k
    if dt is None:
        dt = 0.1 / nu
    cfg = _base_cfg(l0=1, m0=0, nump=nump, numx=nx, numy=1, pmin=pmin, pmax=pmax, xmin=0.0,
                    xmax=L * (nx - 1) / nx, dt=dt, small_dt=dt / ee_substeps, density_np=density,
                    precision=precision)
    p = p_axis(nump, pmin, pmax)
    x = np.arange(nx) * (L / nx)
    T = vth * np.sqrt(1.0 + 1e-3 * np.sin(k * x))
    f = np.zeros((2, 1, nx, nump), np.complex128)
    f[0, 0] = maxwellian(p[None, :], T[:, None])
    fields = np.zeros((6, 1, nx), np.complex128)
    meta = dict(workload="relax1d", nx=nx, np=nump, lmax=1, klambda_ei=klam_ei, nu_ei=nu)
    return cfg, f, fields, meta


def density_for_nu(nu: float, vth: float) -> float:
    """Electron density (1/cm^3) whose collision frequency at v_th is nu (in
    w_p): the inverse of relax1d's nu = 8 re kp / v_th^3, kp = sqrt(4 pi n re)."""
    re = 2.8179402894e-13
    kp = nu * vth ** 3 / (8.0 * re)
    return kp * kp / (4.0 * np.pi * re)


def batch_problems(n: int = 512, seed: int = 2024, precision: int = 1, vth: float = 0.05, klam: float = 0.3):
    """Independent 1D problems of uneven size: nx in [32, 512], np in [32,
    256] and lmax in [1, 16] drawn log-uniform from `seed` and rounded (np to
    a multiple of 4, the bulk copies' 16-byte rule for FP32 rows), each a
    Maxwellian with a density perturbation of amplitude 1e-3 and random phase
    over L = 2 pi/k, k lambda_D = 0.3, np to 8 v_th, nu/w_p uniform in
    [0, 1e-2] (one problem in eight collisionless, nu = 0), FP32 bulk.  dt =
    min(0.05, 0.5 dx/v_max) keeps the explicit advection stable.
    Returns [(cfg, f, fields, collide)], meta."""
    rng = np.random.default_rng(seed)
    k = klam / vth
    L = 2.0 * np.pi / k
    pmax = 8.0 * vth
    vmax = pmax / np.sqrt(1 + pmax * pmax)
    out = []
    ncoef = 0
    for i in range(n):
        nx = int(round(np.exp(rng.uniform(np.log(32), np.log(512)))))
        nump = int(round(np.exp(rng.uniform(np.log(32), np.log(256))) / 4.0)) * 4
        l0 = int(round(np.exp(rng.uniform(np.log(1), np.log(16)))))
        phase = rng.uniform(0, 2 * np.pi)
        nu = 0.0 if i % 8 == 7 else rng.uniform(0.0, 1e-2)
        dx = L / nx
        dt = min(0.05, 0.5 * dx / vmax)
        pmin = pmax / (2.0 * nump)
        density = density_for_nu(nu, vth) if nu > 0 else 1e21
        # small_dt above dt: one e-e substep per step (the reference takes floor(dt/small_dt) + 1)
        cfg = _base_cfg(l0=l0, m0=0, nump=nump, numx=nx, numy=1, pmin=pmin, pmax=pmax, xmin=0.0,
                        xmax=L * (nx - 1) / nx, dt=dt, small_dt=1.5 * dt, density_np=density, precision=precision)
        p = p_axis(nump, pmin, pmax)
        x = np.arange(nx) * dx
        dens = 1.0 + 1e-3 * np.cos(k * x + phase)
        f = np.zeros((num_harmonics(l0, 0), 1, nx, nump), np.complex128)
        f[0, 0] = dens[:, None] * maxwellian(p[None, :], vth)
        fields = np.zeros((6, 1, nx), np.complex128)
        fields[0, 0] = -1e-3 / k * np.sin(k * x + phase)
        out.append((cfg, f, fields, nu > 0))
        ncoef += nx * nump * (l0 + 1)
    meta = dict(workload=f"batch{n}", problems=n, seed=seed, coefficients=ncoef)
    return out, meta


def sensitivity1d(nx: int = 512, l0: int = 2, nump: int = 128, vth: float = 0.05, seed: int = 11,
                  nu_dt: float = 0.05, dt: float = 0.5, length: float = 100.0, ee_substeps: int = 5):
    """Sensitivity configuration: 1D periodic, nx = 512 cells over `length`
    (c/w_p), lmax = 2, np = 128 to 8 v_th, uniform density, T(x) = T0 (1 + 0.2
    g(x)) with g a seeded smooth random field of 8 Fourier modes (max |g| =
    1), nu_ei dt = 0.05 (the density that gives that nu at v_th), dt = 0.5/w_p
    (explicit advection stable: v_max dt/dx < 1), small_dt = dt/5 (the
    explicit e-e step stable).  Returns cfg, the relative temperature tau(x) =
    T/T0, meta."""
    nu = nu_dt / dt
    pmax = 8.0 * vth
    pmin = pmax / (2.0 * nump)
    cfg = _base_cfg(l0=l0, m0=0, nump=nump, numx=nx, numy=1, pmin=pmin, pmax=pmax, xmin=0.0,
                    xmax=length * (nx - 1) / nx, dt=dt, small_dt=dt / ee_substeps,
                    density_np=density_for_nu(nu, vth), precision=0)
    rng = np.random.default_rng(seed)
    x = np.arange(nx) * (length / nx)
    g = np.zeros(nx)
    for k in range(1, 9):
        g += rng.standard_normal() / k * np.cos(2.0 * np.pi * k * x / length + rng.uniform(0, 2 * np.pi))
    g /= np.max(np.abs(g))
    tau = 1.0 + 0.2 * g
    meta = dict(workload="sensitivity1d", nx=nx, lmax=l0, np=nump, nu_ei=nu, vth=vth, seed=seed)
    return cfg, tau, meta


def sensitivity_state(cfg: dict, tau, vth: float = 0.05):
    """plane-layout FP64 state (torch, on tau's device) of a Maxwellian of
    temperature vth^2 tau(x) per cell (Setup_Y::Gaussian_p, OSHUN-1/
    def-Setup.cpp:500-533), f_l = 0 for l >= 1, no fields; differentiable in tau"""
    import torch
    nx, np_, l0 = cfg["numx"], cfg["nump"], cfg["l0"]
    p = torch.tensor(p_axis(np_, cfg["pmin"], cfg["pmax"]), dtype=torch.float64, device=tau.device)
    pt2 = (vth * vth) * tau[:, None]
    f00 = torch.exp(-(p[None, :] ** 2) / (2.0 * pt2)) / ((2.0 * np.pi) ** 1.5 * pt2 ** 1.5)
    rest = torch.zeros(l0 * nx * np_ + 6 * nx, dtype=torch.float64, device=tau.device)
    return torch.cat([f00.reshape(-1), rest])


def build(name: str, precision: int = 0):
    if name not in WORKLOADS:
        raise KeyError(name)
    return globals()[name](precision=precision)
