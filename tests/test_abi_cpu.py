"""C ABI checks that need no GPU: the library builds, loads, exports every
symbol include/oshun_b200.h declares, and fails loudly (a status code, no
CPU fallback) where a device is needed."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "oshun_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|long long|const char\*)\s+(oshun_\w+)\s*\(", src, re.M)))


@pytest.fixture(scope="module")
def lib():
    from oshun_b200 import build as b
    b.build()
    from oshun_b200 import abi
    return abi.load()


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "oshun_create" in syms and "oshun_step" in syms and len(syms) >= 18


def test_library_exports_every_declared_symbol(lib):
    from oshun_b200 import abi
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert set(declared_symbols()) == set(abi.EXPORTED)


def test_abi_version(lib):
    assert lib.oshun_abi_version() == 1


def _cfg(**over):
    from oshun_b200.abi import make_cfg
    kw = dict(l0=3, m0=2, nump=16, numx=8, numy=1, pmin=0.0125, pmax=0.4, xmin=0.0, xmax=1.0, dt=0.05)
    kw.update(over)
    return make_cfg(**kw)


@pytest.mark.parametrize("over,code", [
    (dict(m0=4), 1),                 # m0 > l0
    (dict(nump=2), 1),               # too few momentum cells
    (dict(dt=0.0), 1),               # no step
    (dict(l0=12, m0=9), 2),          # m0 above the compiled maximum
    (dict(precision=7), 1),
])
def test_create_rejects_bad_config(lib, over, code):
    h = ctypes.c_void_p()
    rc = lib.oshun_create(ctypes.byref(_cfg(**over)), ctypes.byref(h))
    assert rc == code
    assert not h.value
    assert len(lib.oshun_last_error()) > 0


def test_create_without_device_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = lib.oshun_create(ctypes.byref(_cfg()), ctypes.byref(h))
    assert rc == 6  # OSHUN_ERR_NO_DEVICE
    assert not h.value


def test_null_handles_rejected(lib):
    assert lib.oshun_rk4_step(None) == 1
    assert lib.oshun_destroy(None) == 1
    assert lib.oshun_upload(None, None, None) == 1
