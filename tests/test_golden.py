"""The C restatement against the reference's own outputs (tests/golden,
generated by tests/golden/make_golden.py from the OSHUN-1 sources)."""
import json
import os

import pytest

from oracle.cases import read_case
from tests.gpu_util import worst_rel

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))
TOL = 1e-12  # relative L2 per harmonic and per field, FP64


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_oracle_matches_reference_golden(oracle, name):
    st = read_case(os.path.join(GOLDEN, name + ".in.case"))
    ref = read_case(os.path.join(GOLDEN, name + ".out.case"))
    out = st
    for op in MANIFEST[name]["ops"]:
        if op == "rhs":
            out = oracle.rhs(out)
        else:
            parts = op.split(":")
            out = oracle.steps(out, int(parts[1]), int(parts[2]) if len(parts) > 2 else 15)
    err, where = worst_rel(out, ref)
    assert err <= TOL, (name, err, where)


def test_golden_cases_move(oracle):
    """Every golden case changes its input well beyond the tolerance, so a
    checker that did nothing could not pass."""
    for name in MANIFEST:
        st = read_case(os.path.join(GOLDEN, name + ".in.case"))
        ref = read_case(os.path.join(GOLDEN, name + ".out.case"))
        err, _ = worst_rel(st, ref)
        assert err > 1e-6, name
