import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built liboshun_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.cases import Oracle, ORACLE_SO
    if not os.path.exists(ORACLE_SO):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "liboshun_oracle.so")],
                       check=True, capture_output=True)
    orc = Oracle()
    yield orc
    orc.set_yadv_chain(True)
    orc.set_ee_implicit(0)
    orc.set_mirror_x(False)
