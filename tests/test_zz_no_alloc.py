"""The allocation-free collision entry point (oshun_collide_flm_noalloc).

It serves callers that cannot allocate device memory inside their time loop
-- an application whose device memory all belongs to its own pool, or a
foreign runtime that owns every device buffer -- by keeping its scratch in a
fixed __device__ array.  This file is collected last, so a run that stops at
its first failure has already run every other test; it passes alone in a
fresh process (the first call does the per-device set-up) and after the
others (the shared scratch keeps the previous call's contents).
"""
import ctypes

import numpy as np
import pytest

from oracle.cases import Deck, seeded_state
from tests.gpu_util import cfg_of

pytestmark = pytest.mark.gpu
TOL = 1e-12   # relative L2 per harmonic, the bar of the FP64 parity tests


@pytest.mark.parametrize("tri", [0, 1])
def test_noalloc_matches_handle_entry_points(tri):
    from oshun_b200 import Handle, abi
    lib = abi.load()
    d = Deck(l0=4, m0=2, nump=24, numx=4, numy=3, if_implicit1D=0, if_tridiagonal=tri,
             dt=0.3, small_dt=0.1, density_np=1e25, xmax=2.0, ymax=3.0)
    st = seeded_state(d, seed=31)
    kw = cfg_of(d)

    # two implicit steps through the existing entry points (Euler_Backward::advance_1/_lm)
    with Handle(**kw) as h:
        h.upload(st.f, st.fields)
        t = 0.0
        for _ in range(2):
            t += d.dt
            h.collide_f1(t)
            h.collide_flm(t)
        fa, fla = h.download()

    # the same two steps, twice in a row, through the allocation-free entry point on
    # device buffers owned by the caller (here a second handle's state)
    with Handle(**kw) as h2:
        h2.upload(st.f, st.fields)
        h2.synchronize()
        f00, planes, _, _, _ = h2.device_state()
        cfg = abi.make_cfg(**kw)
        t_prev, t = 0.0, 0.0
        for _ in range(2):
            t += d.dt
            count = ctypes.c_longlong(-1)
            flags = ctypes.c_int(-1)
            rc = lib.oshun_collide_flm_noalloc(ctypes.byref(cfg), ctypes.c_void_p(f00), ctypes.c_void_p(planes),
                                               t - t_prev, None, ctypes.byref(count), ctypes.byref(flags))
            assert rc == 0, lib.oshun_last_error().decode()
            assert count.value == 0 and flags.value == 0, (count.value, flags.value)
            t_prev = t
        h2.synchronize()
        fb, flb = h2.download()

    for (l, m) in d.harmonics():
        a, b = fa[d.ind(l, m)], fb[d.ind(l, m)]
        err = np.linalg.norm(b - a) / max(np.linalg.norm(a), 1e-300)
        assert err <= TOL, ((l, m), err)
    assert np.array_equal(fla, flb)


@pytest.mark.parametrize("tri", [0, 1])
def test_noalloc_matches_oracle(oracle, tri):
    """One implicit step (f1 then f_lm, Euler_Backward::advance_1/_lm,
    OSHUN-1/def-FokkerPlanck.cpp:1270-1304) against the C restatement."""
    from oshun_b200 import Handle, abi
    from oracle.cases import State
    from tests.gpu_util import worst_rel
    lib = abi.load()
    d = Deck(l0=5, m0=3, nump=40, numx=5, numy=3, if_implicit1D=0, if_tridiagonal=tri,
             dt=0.3, small_dt=0.1, density_np=1e25, xmax=2.0, ymax=3.0)
    st = seeded_state(d, seed=33)
    kw = cfg_of(d)
    with Handle(**kw) as h:
        h.upload(st.f, st.fields)
        h.synchronize()
        f00, planes, _, _, _ = h.device_state()
        cfg = abi.make_cfg(**kw)
        for _ in range(2):   # the second call finds the first one's tables in the scratch
            h.upload(st.f, st.fields)
            h.synchronize()
            flags = ctypes.c_int(-1)
            rc = lib.oshun_collide_flm_noalloc(ctypes.byref(cfg), ctypes.c_void_p(f00), ctypes.c_void_p(planes),
                                               d.dt, None, None, ctypes.byref(flags))
            assert rc == 0, lib.oshun_last_error().decode()
            assert flags.value == 0
            f, fl = h.download()
            err, where = worst_rel(State(d, f, fl), oracle.steps(st, 1, 12))
            assert err <= TOL, (err, where)


def test_noalloc_reports_nan():
    """A NaN in the planes comes back as bit 1 and OSHUN_ERR_NUMERIC."""
    from oshun_b200 import Handle, abi
    lib = abi.load()
    d = Deck(l0=3, m0=1, nump=32, numx=4, numy=2, if_implicit1D=0, if_tridiagonal=1,
             dt=0.3, small_dt=0.1, density_np=1e25, xmax=2.0, ymax=3.0)
    st = seeded_state(d, seed=34)
    st.f[d.ind(2, 1), 1, 3, 7] = complex(np.nan, 0.0)
    kw = cfg_of(d)
    with Handle(**kw) as h:
        h.upload(st.f, st.fields)
        h.synchronize()
        f00, planes, _, _, _ = h.device_state()
        cfg = abi.make_cfg(**kw)
        flags = ctypes.c_int(-1)
        rc = lib.oshun_collide_flm_noalloc(ctypes.byref(cfg), ctypes.c_void_p(f00), ctypes.c_void_p(planes),
                                           d.dt, None, None, ctypes.byref(flags))
        assert rc == 5 and flags.value & 2, (rc, flags.value)


def test_noalloc_rejects_oversize():
    from oshun_b200 import abi
    lib = abi.load()
    d = Deck(l0=80, m0=2, nump=24, numx=4, numy=1)
    cfg = abi.make_cfg(**cfg_of(d))
    rc = lib.oshun_collide_flm_noalloc(ctypes.byref(cfg), ctypes.c_void_p(16), ctypes.c_void_p(16), 0.1, None, None,
                                       None)
    assert rc == 2   # OSHUN_ERR_UNSUPPORTED, before any device work
    assert b"l0 <= 64" in lib.oshun_last_error()
