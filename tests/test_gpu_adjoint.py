"""Adjoint of the small step (oshun_adjoint_*, 1D, m0 = 0, FP64) and the
checkpointed torch.autograd.Function of oshun_b200.adjoint.

* one step's VJP against central differences of the production forward:
  <lam, (step(y + e d) - step(y - e d)) / 2e> = <vjp(y, lam), d>, with and
  without the collision step (the five fields other than E_x carry no
  cotangent and no perturbation: with m0 = 0 they never act on f or E_x);
* the gradient of the time-integrated heat flux of one cell with respect to
  every cell's initial temperature, through checkpointed segments, against
  central differences (h = 1e-4 on T/T0) of the GPU forward and of the C
  restatement of the reference's algorithm (the FP64 reference gradient),
  and independent of the checkpoint spacing;
* the sensitivity configuration at full size (nx = 512, lmax = 2, np = 128,
  500 steps, checkpoints every 50, heat flux at cell 256) against central
  differences on 16 seeded components;
* the FP32 bulk form (l >= 1 planes and fields in FP32, the stage transposes
  in FP32 arithmetic, f00 and the collision transposes in FP64) against the
  FP64 gradient: every component within 1e-4 of the largest;
* the general transpose (2D grids, m0 > 0: every E, B, advection, current
  and Maxwell coupling, the collided m > 0 planes): one step's VJP against
  central differences of the production forward, 2D and 1D with m0 = 2,
  with and without collisions.
Gradient bar: max |g_i - fd_i| <= 1e-5 max |fd|.
"""
import numpy as np
import pytest

from oracle.cases import Deck, State

pytestmark = pytest.mark.gpu
H = 1e-4


def _small_cfg(nx=32, np_=32, l0=2):
    from oshun_b200 import workloads
    cfg, tau, meta = workloads.sensitivity1d(nx=nx, l0=l0, nump=np_, length=100.0 * nx / 512)
    return cfg, tau


def _run(cfg):
    from oshun_b200.adjoint import Run
    return Run(**cfg)


def _loss(run, cfg, tau_t, nsteps, every, cell, grad=False):
    import torch
    from oshun_b200 import workloads
    from oshun_b200.adjoint import StepsWithCheckpoints, heat_flux_weight
    w = heat_flux_weight(cfg, cell)
    if grad:
        tau_t = tau_t.clone().requires_grad_(True)
        y0 = workloads.sensitivity_state(cfg, tau_t)
        Q = StepsWithCheckpoints.apply(y0, run, nsteps, every, w)
        Q.backward()
        return float(Q.detach()), tau_t.grad.detach().cpu().numpy()
    with torch.no_grad():
        y0 = workloads.sensitivity_state(cfg, tau_t)
        return float(StepsWithCheckpoints.apply(y0, run, nsteps, every, w)), None


@pytest.mark.parametrize("collisions", [False, True])
def test_step_vjp_directional(collisions):
    import torch
    from oshun_b200 import workloads
    from oshun_b200.adjoint import state_layout
    cfg, tau = _small_cfg(nx=16)
    run = _run(cfg)
    lay = state_layout(cfg)
    gen = torch.Generator(device="cuda").manual_seed(3)
    y = workloads.sensitivity_state(cfg, torch.tensor(tau, device="cuda"))
    f = y[lay["f"]].view(lay["fshape"])
    scale = f[0].abs().max()
    f[1:] = 0.05 * scale * torch.randn(f[1:].shape, generator=gen, device="cuda", dtype=torch.float64)
    y[lay["fields"]][: cfg["numx"]] = 1e-3 * torch.randn(cfg["numx"], generator=gen, device="cuda", dtype=torch.float64)
    d = torch.zeros_like(y)
    d[lay["f"]] = 1e-2 * scale * torch.randn(lay["f"].stop, generator=gen, device="cuda", dtype=torch.float64)
    d[lay["f"]].view(lay["fshape"])[0] *= 0.1          # f00 perturbation small against f00
    d[lay["fields"]][: cfg["numx"]] = 1e-4 * torch.randn(cfg["numx"], generator=gen, device="cuda", dtype=torch.float64)
    lam = torch.zeros_like(y)
    lam[lay["f"]] = torch.randn(lay["f"].stop, generator=gen, device="cuda", dtype=torch.float64)
    lam[lay["fields"]][: cfg["numx"]] = torch.randn(cfg["numx"], generator=gen, device="cuda", dtype=torch.float64)
    clocks = (0.0, 0.0, 0.0)
    eps = 1e-3
    yp = run.forward(y + eps * d, clocks, collisions)
    ym = run.forward(y - eps * d, clocks, collisions)
    lhs = float(torch.dot(lam, yp - ym)) / (2 * eps)
    rhs = float(torch.dot(run.vjp(y, lam, clocks, collisions), d))
    assert abs(lhs - rhs) <= 1e-7 * (abs(lhs) + abs(rhs)), (lhs, rhs)


def _oracle_loss(oracle, cfg, tau, nsteps, cell):
    """the same functional through the C restatement (the reference's algorithm)"""
    from oshun_b200 import workloads
    from oshun_b200.adjoint import heat_flux_weight
    d = Deck(l0=cfg["l0"], m0=0, nump=cfg["nump"], numx=cfg["numx"], numy=1, pmin=cfg["pmin"], pmax=cfg["pmax"],
             xmin=cfg["xmin"], xmax=cfg["xmax"], dt=cfg["dt"], small_dt=cfg["small_dt"],
             density_np=cfg["density_np"])
    st = State(d)
    p = d.pr()
    st.f[0, 0] = workloads.maxwellian(p[None, :], 0.05 * np.sqrt(tau)[:, None])
    w = heat_flux_weight(cfg, cell, device="cpu").numpy()
    nx, np_ = cfg["numx"], cfg["nump"]
    w1 = w[(1 * nx + cell) * np_:(1 * nx + cell + 1) * np_]
    Q = 0.0
    for _ in range(nsteps):
        st = oracle.steps(st, 1, 15)
        Q += cfg["dt"] * float(np.dot(w1, st.f[1, 0, cell].real))
    return Q


def test_checkpointed_gradient_small(oracle):
    import torch
    cfg, tau = _small_cfg()
    run = _run(cfg)
    nsteps, cell = 30, 16
    tt = torch.tensor(tau, device="cuda")
    Q, g = _loss(run, cfg, tt, nsteps, 7, cell, grad=True)
    _, g1 = _loss(run, cfg, tt, nsteps, 1000, cell, grad=True)     # no intermediate checkpoint
    assert np.max(np.abs(g - g1)) <= 1e-12 * np.max(np.abs(g))
    comps = [0, 5, 11, 16, 17, 30]
    fd, fd_ref = [], []
    for i in comps:
        e = np.zeros_like(tau)
        e[i] = H
        qp, _ = _loss(run, cfg, torch.tensor(tau + e, device="cuda"), nsteps, 7, cell)
        qm, _ = _loss(run, cfg, torch.tensor(tau - e, device="cuda"), nsteps, 7, cell)
        fd.append((qp - qm) / (2 * H))
        fd_ref.append((_oracle_loss(oracle, cfg, tau + e, nsteps, cell) -
                       _oracle_loss(oracle, cfg, tau - e, nsteps, cell)) / (2 * H))
    fd, fd_ref = np.array(fd), np.array(fd_ref)
    scale = np.max(np.abs(fd))
    assert scale > 0
    assert np.max(np.abs(g[comps] - fd)) <= 1e-5 * scale, (g[comps], fd)
    assert np.max(np.abs(g[comps] - fd_ref)) <= 1e-5 * scale, (g[comps], fd_ref)


@pytest.mark.parametrize("prec", [0, 1])
def test_gradient_on_a_torch_stream_matches_waiting_form(prec):
    """On a non-default torch stream the handle's calls are queued on that
    stream without waiting: the loss and gradient are bitwise those of the
    waiting form (same kernels, same order), and a second run on the same
    stream reproduces them."""
    import torch
    cfg, tau = _small_cfg()
    cfg = dict(cfg, precision=prec)
    tt = torch.tensor(tau, device="cuda")
    run0 = _run(cfg)
    q0, g0 = _loss(run0, cfg, tt, 30, 7, 16, grad=True)     # default stream: every call waits
    run0.close()
    run1 = _run(cfg)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        q1, g1 = _loss(run1, cfg, tt, 30, 7, 16, grad=True)
        q2, g2 = _loss(run1, cfg, tt, 30, 7, 16, grad=True)
    torch.cuda.synchronize()
    run1.close()
    assert q1 == q0 and q2 == q0, (q0, q1, q2)
    assert np.array_equal(g1, g0) and np.array_equal(g2, g0)


def test_sensitivity_full_size():
    import torch
    from oshun_b200 import workloads
    cfg, tau, meta = workloads.sensitivity1d()
    run = _run(cfg)
    nsteps, every, cell = 500, 50, 256
    tt = torch.tensor(tau, device="cuda")
    Q, g = _loss(run, cfg, tt, nsteps, every, cell, grad=True)
    comps = sorted(np.random.default_rng(2024).choice(cfg["numx"], 16, replace=False).tolist())
    fd = []
    for i in comps:
        e = np.zeros_like(tau)
        e[i] = H
        qp, _ = _loss(run, cfg, torch.tensor(tau + e, device="cuda"), nsteps, every, cell)
        qm, _ = _loss(run, cfg, torch.tensor(tau - e, device="cuda"), nsteps, every, cell)
        fd.append((qp - qm) / (2 * H))
    fd = np.array(fd)
    scale = np.max(np.abs(fd))
    assert scale > 0 and np.isfinite(g).all()
    assert np.max(np.abs(g[comps] - fd)) <= 1e-5 * scale, (g[comps], fd)


def test_fp32_bulk_gradient_against_fp64():
    import torch
    cfg, tau = _small_cfg()
    nsteps, cell = 30, 16
    tt = torch.tensor(tau, device="cuda")
    _, g64 = _loss(_run(cfg), cfg, tt, nsteps, 7, cell, grad=True)
    _, g32 = _loss(_run(dict(cfg, precision=1)), cfg, tt, nsteps, 7, cell, grad=True)
    scale = np.max(np.abs(g64))
    assert scale > 0 and np.isfinite(g32).all()
    err = np.max(np.abs(g32 - g64)) / scale
    assert err <= 1e-4, err
    assert err > 0.0    # the FP32 form does run in FP32


def _plane_vector(d, st):
    """the state in the plane layout of the adjoint vectors"""
    import torch
    from oshun_b200 import Handle
    from tests.gpu_util import cfg_of
    cells = d.numx * d.numy
    with Handle(**cfg_of(d)) as h:
        qs = {(l, m): h.plane_index(l, m) for (l, m) in d.harmonics() if l >= 1}
    nplanes = sum(2 if m > 0 else 1 for (l, m) in d.harmonics() if l >= 1)
    ps = cells * d.nump
    v = np.zeros((1 + nplanes) * ps + 6 * cells)
    v[:ps] = st.f[d.ind(0, 0)].real.reshape(-1)
    for (l, m), q in qs.items():
        h = st.f[d.ind(l, m)]
        v[(1 + q) * ps:(2 + q) * ps] = h.real.reshape(-1)
        if m > 0:
            v[(2 + q) * ps:(3 + q) * ps] = h.imag.reshape(-1)
    v[(1 + nplanes) * ps:] = st.fields.real.reshape(-1)
    return torch.tensor(v, device="cuda")


@pytest.mark.parametrize("collisions", [False, True])
@pytest.mark.parametrize("ny", [4, 1])
def test_step_vjp_directional_general(collisions, ny):
    import torch
    from oracle.cases import seeded_state
    from tests.gpu_util import cfg_of
    d = Deck(l0=3, m0=2, nump=32, numx=6, numy=ny, if_implicit1D=0, if_tridiagonal=1, dt=0.1, small_dt=0.05,
             density_np=1e25, xmax=2.0, ymax=3.0)
    st = seeded_state(d, seed=51, fields=True)
    run = _run(cfg_of(d))
    y = _plane_vector(d, st)
    assert y.numel() == run.n
    gen = torch.Generator(device="cuda").manual_seed(5)
    ps = d.numx * d.numy * d.nump
    scale = float(y[:ps].abs().max())
    d_ = 1e-3 * scale * torch.randn(run.n, generator=gen, device="cuda", dtype=torch.float64)
    d_[:ps] *= 0.1
    nf = 6 * d.numx * d.numy
    d_[-nf:] = 1e-5 * torch.randn(nf, generator=gen, device="cuda", dtype=torch.float64)
    lam = torch.randn(run.n, generator=gen, device="cuda", dtype=torch.float64)
    clocks = (0.0, 0.0, 0.0)
    eps = 1e-3
    yp = run.forward(y + eps * d_, clocks, collisions)
    ym = run.forward(y - eps * d_, clocks, collisions)
    lhs = float(torch.dot(lam, yp - ym)) / (2 * eps)
    rhs = float(torch.dot(run.vjp(y, lam, clocks, collisions), d_))
    assert abs(lhs - rhs) <= 1e-7 * (abs(lhs) + abs(rhs)), (lhs, rhs)
