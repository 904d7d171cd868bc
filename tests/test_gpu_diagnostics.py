"""Device moments and restart files through the C ABI, against the
reference's own code in the checker build (oracle/_ref):

* oshun_moments against the files Parallel_Output::nonrelativistic_moments
  writes (OSHUN-1/def-Parallel.cpp:1677-2258; Export_mom prints each float
  with 10 digits, def-Export.cpp:405-470);
* oshun_restart_write / _read against Restart_Facility (def-Export.cpp:
  733-836): identical bytes, and a run resumed from the reference's file
  continues as the reference does.
"""
import os
import tempfile

import numpy as np
import pytest

from oracle.cases import Deck, State, seeded_state
from tests.gpu_util import cfg_of, run_gpu, worst_rel
from tests.test_restart import run_ref_in

pytestmark = pytest.mark.gpu

# moment -> file written by the reference (OUTPUT/MOM/<dir>/<stem>_<step:05>.txt)
FILES = {"Vx": "Vx/Vx", "Vy": "Vy/Vy", "VxVx": "VxVx/VxVx", "VyVy": "VyVy/VyVy", "VzVz": "VzVz/VzVz",
         "VxVy": "VxVy/VxVy", "VxVz": "VxVz/VxVz", "VyVz": "VyVz/VyVz", "Vsq": "Vsq/Vsq", "T_eV": "T_eV/T",
         "P_Mbar": "P_Mbar/P", "ND": "ND/ND", "Nu": "Nu/nu", "Qx": "Qx/Qx", "Kx": "Qx/Kx", "Qy": "Qy/Qy",
         "Ky": "Qy/Ky"}
MOM_TOL = 2e-6   # relative L2 per moment (float results; a few ulps)


def reference_moments(st, step=3):
    with tempfile.TemporaryDirectory() as td:
        for stem in FILES.values():
            os.makedirs(os.path.join(td, "OUTPUT", "MOM", stem.split("/")[0]), exist_ok=True)
        run_ref_in(td, st, [f"moments:{step}"])
        out = {}
        for name, stem in FILES.items():
            vals = open(os.path.join(td, "OUTPUT", "MOM", f"{stem}_{step:05d}.txt")).read().split("\n")
            n1, n2 = int(vals[4]), int(vals[5])
            data = np.array([float(v) for v in vals[6 + n1 + n2:6 + n1 + n2 + n1 * n2]], np.float64)
            out[name] = data.reshape(n2, n1)     # x fastest
    return out


def _real_1d(st):
    for (l, m) in st.deck.harmonics():
        if m > 0:
            st.f[st.deck.ind(l, m)] = 0
    st.fields[1:] = 0
    return st


@pytest.mark.parametrize("kw", [dict(l0=4, m0=2, nump=24, numx=6, numy=5), dict(l0=3, m0=3, nump=40, numx=4, numy=4),
                                dict(l0=5, m0=2, nump=32, numx=8, numy=1)])
@pytest.mark.parametrize("steps", [0, 1])
def test_moments_match_reference_output(kw, steps):
    from oshun_b200 import Handle
    d = Deck(xmax=2.0, ymax=3.0, if_implicit1D=1 if kw["numy"] == 1 else 0, dt=0.1, small_dt=0.05,
             density_np=1e25, **kw)
    st = seeded_state(d, seed=51, fields=d.numy > 1)
    if d.numy == 1:
        st = _real_1d(st)
    if steps:
        st = run_gpu(st, [f"step:{steps}:15"], fast_path=True)
    ref = reference_moments(st)
    with Handle(**cfg_of(d)) as h:
        h.upload(st.f, st.fields)
        mom = h.moments()
    names = Handle.MOMENTS
    worst = {}
    for name, want in ref.items():
        got = mom[names.index(name)].astype(np.float64)
        if d.numy == 1:                         # the checker runs 1D decks on 4 identical rows
            got = np.repeat(got, want.shape[0], axis=0)
        den = np.linalg.norm(want)
        worst[name] = float(np.linalg.norm(got - want) / den) if den > 0 else float(np.linalg.norm(got))
    bad = {k: v for k, v in worst.items() if not v <= MOM_TOL}
    assert not bad, (bad, worst)


def test_restart_write_read_through_handle():
    from oshun_b200 import Handle
    from oshun_b200.abi import restart_pack
    d = Deck(l0=4, m0=2, nump=24, numx=5, numy=4, xmax=2.0, ymax=3.0, if_implicit1D=0, dt=0.2, small_dt=0.1,
             density_np=1e25)
    st = seeded_state(d, seed=52)
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, "re")
        with Handle(**cfg_of(d)) as h:
            h.upload(st.f, st.fields)
            h.step(1, collisions=True)
            f, fl = h.download()
            h.restart_write(prefix, 0, 1, 4)
        img = open(prefix + "_000000_001.dat", "rb").read()
        assert img == restart_pack(cfg_of(d), f, fl, 4)
        with Handle(**cfg_of(d)) as h2:
            h2.restart_read(prefix, 0, 1, 4)
            f2, fl2 = h2.download()
    assert np.array_equal(f2, f) and np.array_equal(fl2, fl)


def test_resume_from_reference_restart_file():
    """The reference writes its state after one step; a handle reads that
    file and takes the second step; the reference's own two steps agree at
    the FP64 bar."""
    from oshun_b200 import Handle
    d = Deck(l0=4, m0=2, nump=24, numx=5, numy=4, xmax=2.0, ymax=3.0, if_implicit1D=0, dt=0.2, small_dt=0.1,
             density_np=1e25)
    st = seeded_state(d, seed=53)
    with tempfile.TemporaryDirectory() as td:
        run_ref_in(td, st, ["step:1:15", "restart_write:0:1"])
        two = run_ref_in(td, st, ["step:2:15"])
        cfg = cfg_of(d)
        cfg["t0"] = d.dt       # the resumed run's clocks start at the file's time
        with Handle(**cfg) as h:
            h.restart_read(os.path.join(td, "RESTART", "re"), 0, 1, 4)
            h.step(1, collisions=True)
            f, fl = h.download()
    err, where = worst_rel(State(d, f, fl), two)
    assert err <= 1e-12, (err, where)
