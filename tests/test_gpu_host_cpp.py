"""The C++ host layer (oshun_b200/host/oshun.hpp) driving the C ABI in the
reference's main-loop order, checked against the reference's own outputs
(tests/golden)."""
import json
import os
import subprocess
import tempfile

import pytest

from oracle.cases import read_case
from tests.gpu_util import worst_rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))
DRIVER = os.path.join(ROOT, "oshun_b200", "host", "oshun_main_loop")
STEP_CASES = sorted(n for n, v in MANIFEST.items() if v["ops"][0].startswith("step:"))
TOL = 1e-12


def _driver():
    if not os.path.exists(DRIVER):
        from oshun_b200 import build
        build.build()
    return DRIVER


def test_driver_usage_and_missing_device():
    """Without arguments the driver prints its usage; without a GPU it fails
    with the C ABI's no-device status instead of computing anything."""
    r = subprocess.run([_driver()], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    name = STEP_CASES[0]
    with tempfile.TemporaryDirectory() as td:
        r = subprocess.run([_driver(), os.path.join(GOLDEN, name + ".in.case"), os.path.join(td, "o.case"), "1"],
                           capture_output=True, text=True)
    assert r.returncode == 3 and "status 6" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", STEP_CASES)
def test_cpp_main_loop_matches_reference(name):
    op = MANIFEST[name]["ops"][0].split(":")
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.case")
        r = subprocess.run([_driver(), os.path.join(GOLDEN, name + ".in.case"), out, op[1], op[2]],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = read_case(out)
    ref = read_case(os.path.join(GOLDEN, name + ".out.case"))
    err, where = worst_rel(got, ref)
    assert err <= TOL, (name, err, where)
