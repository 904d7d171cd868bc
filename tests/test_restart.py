"""Restart files in the reference's byte layout (Restart_Facility::Write and
::Read, OSHUN-1/def-Export.cpp:733-836), checked against the reference's own
restart code in the checker build (oracle/_ref): no device is needed for the
file image (oshun_restart_pack / _unpack)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle.cases import REF_BIN, Deck, State, read_case, reference_available, seeded_state, write_case
from tests.gpu_util import cfg_of

pytestmark = pytest.mark.skipif(not reference_available(), reason="reference checker not built")


def run_ref_in(td, st, ops):
    """The reference checker with `td` as its working directory (its restart
    files live in td/RESTART); returns the state it ends with."""
    os.makedirs(os.path.join(td, "RESTART"), exist_ok=True)
    fin, fout = os.path.join(td, "in.case"), os.path.join(td, "out.case")
    write_case(fin, st)
    r = subprocess.run([REF_BIN, fin, fout] + list(ops), cwd=td, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return read_case(fout)


CASES = [
    dict(l0=4, m0=2, nump=24, numx=5, numy=4),
    dict(l0=3, m0=3, nump=16, numx=7, numy=6),
]


@pytest.mark.parametrize("kw", CASES)
def test_pack_is_the_reference_file(kw):
    from oshun_b200.abi import restart_pack
    d = Deck(xmax=2.0, ymax=3.0, if_implicit1D=0, **kw)
    st = seeded_state(d, seed=41)
    with tempfile.TemporaryDirectory() as td:
        run_ref_in(td, st, ["restart_write:0:5"])
        ref = open(os.path.join(td, "RESTART", "re_000000_005.dat"), "rb").read()
    ours = restart_pack(cfg_of(d), st.f, st.fields, 4)
    assert len(ours) == len(ref)
    assert ours == ref


def test_pack_after_steps_is_the_reference_file(oracle):
    """A state the reference advanced itself, written by the reference and
    by the packer from the same interior: identical bytes."""
    from oshun_b200.abi import restart_pack, restart_unpack
    d = Deck(l0=4, m0=2, nump=20, numx=5, numy=4, xmax=2.0, ymax=3.0, if_implicit1D=0, dt=0.2, small_dt=0.1,
             density_np=1e25)
    st = seeded_state(d, seed=42)
    with tempfile.TemporaryDirectory() as td:
        out = run_ref_in(td, st, ["step:2:15", "restart_write:3:12"])
        ref = open(os.path.join(td, "RESTART", "re_000003_012.dat"), "rb").read()
    assert restart_pack(cfg_of(d), out.f, out.fields, 4) == ref
    f, fl = restart_unpack(cfg_of(d), ref, 4)
    assert np.array_equal(f, out.f) and np.array_equal(fl, out.fields)


def test_reference_reads_packed_file():
    from oshun_b200.abi import restart_pack
    d = Deck(l0=4, m0=2, nump=24, numx=5, numy=4, xmax=2.0, ymax=3.0, if_implicit1D=0)
    st = seeded_state(d, seed=43)
    img = restart_pack(cfg_of(d), st.f, st.fields, 4)
    with tempfile.TemporaryDirectory() as td:
        os.makedirs(os.path.join(td, "RESTART"))
        with open(os.path.join(td, "RESTART", "re_000002_017.dat"), "wb") as fh:
            fh.write(img)
        blank = State(d)
        out = run_ref_in(td, blank, ["restart_read:2:17"])
    assert np.array_equal(out.f, st.f) and np.array_equal(out.fields, st.fields)


def test_1d_layout_and_round_trip():
    """1D: 1 + 2g rows, each the interior row; the interior comes back."""
    from oshun_b200.abi import restart_pack, restart_unpack
    d = Deck(l0=5, m0=0, nump=16, numx=8, numy=1, xmax=2.0)
    st = seeded_state(d, seed=44, fields=False)
    g = 4
    img = np.frombuffer(restart_pack(cfg_of(d), st.f, st.fields, g), np.complex128)
    nxt, nyt = d.numx + 2 * g, 1 + 2 * g
    harm = img[: d.nh * nyt * nxt * d.nump].reshape(d.nh, nyt, nxt, d.nump)
    for row in range(nyt):
        assert np.array_equal(harm[:, row, g:g + d.numx], st.f[:, 0])
    assert np.array_equal(harm[:, g, :g], st.f[:, 0, d.numx - g:])        # periodic x guards
    f, fl = restart_unpack(cfg_of(d), img.tobytes(), g)
    assert np.array_equal(f, st.f) and np.array_equal(fl, st.fields)


def test_rejects_guard_wider_than_grid():
    from oshun_b200 import OshunError
    from oshun_b200.abi import restart_pack
    d = Deck(l0=3, m0=2, nump=16, numx=3, numy=5)
    st = seeded_state(d, seed=45)
    with pytest.raises(OshunError) as ei:
        restart_pack(cfg_of(d), st.f, st.fields, 4)
    assert ei.value.code == 1 or ei.value.code == 2
