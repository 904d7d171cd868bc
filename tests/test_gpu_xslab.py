"""x boundaries and x slabs (oshun_set_x_boundary, oshun_halo_*,
oshun_step_stage; the reference's bndX and Neighbor_Communications,
OSHUN-1/def-Parallel.cpp:1115-1206, 3040-3129):

* a grid stepped as one x slab whose halo columns are its own opposite edge
  columns is bit-identical to the periodic grid (pipelined stage kernel,
  nump = 32, and the global-load kernel, nump = 33);
* the grid split into two x slabs (two handles on one GPU, the halo columns
  exchanged by device copies before every RK4 stage, as the ranks of
  oshun_b200.slab exchange them) is bit-identical to the single grid, with
  collisions;
* mirrored x boundaries against the C restatement with its mirror rule
  ((-1)^(l+m) on f_lm, -1 on Ey, Ez, Bx): relative L2 <= 1e-12; two slabs
  whose end ranks mirror are bit-identical to the mirrored single grid;
* the x-slab handle refuses the whole-step entry points, and FP32 refuses
  the non-periodic modes.
"""
import numpy as np
import pytest

from oracle.cases import Deck, State, seeded_state
from tests.gpu_util import cfg_of, worst_rel

pytestmark = pytest.mark.gpu
XB_PERIODIC, XB_MIRROR, XB_HALO = 0, 1, 2


def _deck(nx=12, np_=32):
    return Deck(l0=4, m0=2, nump=np_, numx=nx, numy=4, if_implicit1D=0, if_tridiagonal=1, dt=0.2, small_dt=0.07,
                density_np=1e25, xmin=0.0, xmax=0.25 * (nx - 1), ymax=3.0)


def _periodic(d, st, nsteps, mode=XB_PERIODIC):
    from oshun_b200 import Handle
    with Handle(**cfg_of(d)) as h:
        h.set_x_boundary(mode)
        h.upload(st.f, st.fields)
        h.step(nsteps, collisions=True)
        return h.download()


def _slabs(d, st, nsteps, world, mirror=False):
    """`world` slab handles on one GPU, halos exchanged by device copies"""
    import torch
    from oshun_b200 import Handle
    from oshun_b200.slab import slab_cfg
    nxl = d.numx // world
    hs = []
    for r in range(world):
        h = Handle(**slab_cfg(cfg_of(d), r, world))
        h.set_x_boundary(XB_HALO)
        sl = slice(r * nxl, (r + 1) * nxl)
        h.upload(np.ascontiguousarray(st.f[:, :, sl, :]), np.ascontiguousarray(st.fields[:, :, sl]))
        hs.append(h)
    n = hs[0].halo_bytes()
    bl = [torch.empty(n, dtype=torch.uint8, device="cuda") for _ in range(world)]
    br = [torch.empty(n, dtype=torch.uint8, device="cuda") for _ in range(world)]
    for _ in range(nsteps):
        for k in (1, 2, 3, 4):
            for r in range(world):
                hs[r].halo_pack(bl[r].data_ptr(), br[r].data_ptr())
            for r in range(world):
                left, right = (r - 1) % world, (r + 1) % world
                hs[r].halo_unpack(br[left].data_ptr(), bl[right].data_ptr())
                if mirror and r == 0:
                    hs[r].halo_mirror_side(0)
                if mirror and r == world - 1:
                    hs[r].halo_mirror_side(1)
            for r in range(world):
                hs[r].step_stage(k, True)
    parts = [h.download() for h in hs]
    for h in hs:
        h.close()
    return np.concatenate([p[0] for p in parts], axis=2), np.concatenate([p[1] for p in parts], axis=2)


@pytest.mark.parametrize("np_", [32, 33])
def test_self_halo_equals_periodic(np_):
    d = _deck(np_=np_)
    st = seeded_state(d, seed=41)
    f0, l0 = _periodic(d, st, 3)
    f1, l1 = _slabs(d, st, 3, 1)
    assert np.array_equal(f0, f1) and np.array_equal(l0, l1)


@pytest.mark.parametrize("np_", [32, 33])
def test_two_slabs_equal_single_grid(np_):
    d = _deck(np_=np_)
    st = seeded_state(d, seed=42)
    f0, l0 = _periodic(d, st, 3)
    f1, l1 = _slabs(d, st, 3, 2)
    assert np.array_equal(f0, f1) and np.array_equal(l0, l1)


def test_mirror_against_oracle(oracle):
    d = _deck()
    st = seeded_state(d, seed=43)
    oracle.set_mirror_x(True)
    try:
        ref = oracle.steps(st, 3, 15)
    finally:
        oracle.set_mirror_x(False)
    f, fl = _periodic(d, st, 3, XB_MIRROR)
    err, where = worst_rel(State(d, f, fl), ref)
    assert err <= 1e-12, (err, where)
    # the mirror is not the periodic grid
    f0, _ = _periodic(d, st, 3)
    assert not np.array_equal(f, f0)


def test_mirrored_slabs_equal_mirrored_grid():
    d = _deck()
    st = seeded_state(d, seed=44)
    f0, l0 = _periodic(d, st, 3, XB_MIRROR)
    f1, l1 = _slabs(d, st, 3, 3, mirror=True)
    assert np.array_equal(f0, f1) and np.array_equal(l0, l1)


def test_slab_refusals():
    from oshun_b200 import Handle, OshunError
    d = _deck()
    with Handle(**cfg_of(d)) as h:
        h.set_x_boundary(XB_HALO)
        with pytest.raises(OshunError):
            h.step(1)
        with pytest.raises(OshunError):
            h.step_stage(2)
    with Handle(**cfg_of(d, precision=1)) as h:
        with pytest.raises(OshunError):
            h.set_x_boundary(XB_MIRROR)
