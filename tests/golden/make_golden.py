"""Generates the golden cases in this folder by running the reference's own
code (oracle/_ref/oshun_ref, built from the OSHUN-1 sources by
oracle/Makefile) on seeded inputs.

    python tests/golden/make_golden.py

Each case is <name>.in.case (input state + deck) and <name>.out.case (the
reference's output), listed with its operator string in manifest.json.
The reference has no tests or fixtures of its own; these files are the
parity pins for the C restatement (tests/test_golden.py) and, through it,
for the CUDA path.
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.cases import Deck, landau_state, run_reference, seeded_state, write_case  # noqa: E402


def zero_m_positive(st):
    d = st.deck
    for (l, m) in d.harmonics():
        if m > 0:
            st.f[d.ind(l, m)] = 0.0
    st.fields[1:] = 0.0
    return st


def cases():
    out = []
    d = Deck(l0=3, m0=2, nump=16, numx=6, numy=1, if_implicit1D=1, if_tridiagonal=1,
             dt=0.5, small_dt=0.2, density_np=1e25, xmax=2.0)
    out.append(("g1d_l3m2_full", zero_m_positive(seeded_state(d, seed=11, fields=False)), ["step:3:15"]))
    d = Deck(l0=4, m0=3, nump=12, numx=4, numy=5, if_implicit1D=0, if_tridiagonal=1,
             dt=0.3, small_dt=0.1, density_np=1e25, xmax=2.0, ymax=3.0)
    out.append(("g2d_l4m3_tri", seeded_state(d, seed=12), ["step:2:15"]))
    d = Deck(l0=6, m0=6, nump=10, numx=4, numy=4, xmax=2.0, ymax=3.0, if_implicit1D=0)
    out.append(("g2d_l6m6_rhs", seeded_state(d, seed=13), ["rhs"]))
    d = Deck(l0=3, m0=2, nump=14, numx=4, numy=4, if_implicit1D=0, if_tridiagonal=0,
             dt=0.3, small_dt=0.1, density_np=1e25, xmax=2.0, ymax=3.0)
    out.append(("g2d_l3m2_dense", seeded_state(d, seed=14), ["step:2:15"]))
    L = 2.0 * 3.141592653589793 / 6.0
    d = Deck(l0=8, m0=2, nump=32, numx=16, numy=1, pmax=0.4, xmin=0.0, xmax=L * 15.0 / 16.0, dt=0.05)
    out.append(("g1d_landau_rk4", landau_state(d, vth=0.05, alpha=1e-3), ["step:20:1"]))
    return out


def main():
    manifest = {}
    for name, st, ops in cases():
        res = run_reference(st, ops)
        write_case(os.path.join(HERE, name + ".in.case"), st)
        write_case(os.path.join(HERE, name + ".out.case"), res)
        manifest[name] = {"ops": ops}
        print(name, ops)
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
