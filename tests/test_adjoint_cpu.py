"""The adjoint math (oshun_b200/csrc/adjoint_math.h) on the CPU: every
transpose against central finite differences of the same file's forward code,
as <lam, J delta> = <J^T lam, delta> for random lam and delta.

* the 1D RHS (E_x couplings through G/H with the reference's momentum ends,
  x advection, CLEAN_LOW_PC, the current) -- bilinear, so the central
  difference is exact up to rounding;
* the collision step of one cell: e-e RK4 substeps alone, the implicit solves
  alone (with the coefficients' dependence on f00), and both.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def lib():
    d = tempfile.mkdtemp()
    so = os.path.join(d, "libadj.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", so, os.path.join(HERE, "adjoint_cpu.cpp")],
                   check=True)
    L = ctypes.CDLL(so)
    dp = ctypes.POINTER(ctypes.c_double)
    i, d_ = ctypes.c_int, ctypes.c_double
    L.ac_collide.argtypes = [i, i, dp, d_, d_, d_, d_, i, dp, dp, i, i, i, d_, d_]
    L.ac_collide_T.argtypes = [i, i, dp, d_, d_, d_, d_, i, dp, dp, i, i, i, d_, d_, dp, dp]
    L.ac_rhs.argtypes = [i, i, i, dp, dp, dp, dp, dp, dp, dp]
    L.ac_vjp.argtypes = [i, i, i, dp, dp, dp, dp, dp, dp, dp, dp, dp]
    return L


def P(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _tables(np_=32, pmax=0.4):
    p = (np.arange(np_) + 0.5) * (pmax / np_)
    v = p / np.sqrt(1 + p * p)
    dv = np.diff(v, prepend=0.0)
    T = np.zeros((12, np_))
    T[0] = v
    T[1, 1:] = 0.5 * v[1:] ** 4 * dv[1:]
    T[2, 1:] = 0.5 * v[:-1] ** 4 * dv[1:]
    T[3, 1:] = 0.5 * v[1:] ** 2 * dv[1:]
    T[4, 1:] = 0.5 * v[:-1] ** 2 * dv[1:]
    T[5, 1:] = 0.5 * v[1:] * dv[1:]
    T[6, 1:] = 0.5 * v[:-1] * dv[1:]
    T[7] = v ** 3
    vh = np.concatenate([[0.0], 0.5 * (v[1:] + v[:-1]), [v[-1]]])
    T[8] = 1.0 / (v * v * np.maximum(np.diff(vh), 1e-12))
    T[9, :-1] = vh[1:-1] ** 2 / np.diff(v)
    T[10] = v ** 5
    T[11] = v ** 7
    return p, v, np.ascontiguousarray(T)


def _coll_case(l0=2, np_=32, seed=0):
    rng = np.random.default_rng(seed)
    p, v, T = _tables(np_)
    vth = 0.05
    f00 = np.exp(-p * p / (2 * vth * vth)) / ((2 * np.pi) ** 1.5 * vth ** 3)
    f00 *= 1 + 0.05 * rng.standard_normal(np_) * np.exp(-p / 0.2)
    fl = 1e-2 * f00[None, :] * rng.standard_normal((l0, np_))
    re = 2.8179402894e-13
    dens = 1e22
    kp = np.sqrt(4 * np.pi * dens * re)
    consts = (dens, 1.0, 4 * np.pi / 3 * re * kp, re * kp)
    return T, f00, np.ascontiguousarray(fl), consts


def _coll(lib, T, f00, fl, consts, l0, ee, eb, nsub, hsub, Dt, NB=4):
    a, b = f00.copy(), fl.copy()
    lib.ac_collide(T.shape[1], NB, P(T), *consts, l0, P(a), P(b), ee, eb, nsub, hsub, Dt)
    return a, b


@pytest.mark.parametrize("ee,eb,nsub", [(1, 0, 1), (1, 0, 3), (0, 1, 1), (1, 1, 2)])
def test_collision_transpose(lib, ee, eb, nsub):
    l0 = 2
    T, f00, fl, consts = _coll_case(l0)
    rng = np.random.default_rng(5)
    # a step of ~0.05 collision times at this density
    hsub, Dt = 40.0, 80.0
    l00 = rng.standard_normal(f00.size)
    ll = rng.standard_normal(fl.shape)
    d00 = rng.standard_normal(f00.size) * f00
    dl = rng.standard_normal(fl.shape) * 1e-2 * f00[None, :]
    eps = 1e-4
    a1, b1 = _coll(lib, T, f00 + eps * d00, fl + eps * dl, consts, l0, ee, eb, nsub, hsub, Dt)
    a0, b0 = _coll(lib, T, f00 - eps * d00, fl - eps * dl, consts, l0, ee, eb, nsub, hsub, Dt)
    lhs = (np.dot(l00, a1 - a0) + np.sum(ll * (b1 - b0))) / (2 * eps)
    lam00, laml = l00.copy(), np.ascontiguousarray(ll.copy())
    lib.ac_collide_T(T.shape[1], 4, P(T), *consts, l0, P(f00), P(fl), ee, eb, nsub, hsub, Dt, P(lam00), P(laml))
    rhs = np.dot(lam00, d00) + np.sum(laml * dl)
    assert abs(lhs - rhs) <= 1e-6 * (abs(lhs) + abs(rhs)), (lhs, rhs)


def test_collision_step_moves(lib):
    """the forward actually changes f at these parameters (the test above is not vacuous)"""
    l0 = 2
    T, f00, fl, consts = _coll_case(l0)
    a, b = _coll(lib, T, f00, fl, consts, l0, 1, 1, 2, 40.0, 80.0)
    assert np.linalg.norm(a - f00) > 1e-4 * np.linalg.norm(f00)
    assert np.linalg.norm(b - fl) > 1e-2 * np.linalg.norm(fl)


def _rhs_case(l0=3, np_=24, nx=7, seed=1):
    rng = np.random.default_rng(seed)
    p = (np.arange(np_) + 0.5) * (0.4 / np_)
    ptab = np.ascontiguousarray(np.stack([1 / p, p / np.sqrt(1 + p * p), 0.01 * p ** 3]))
    coef = np.ascontiguousarray(rng.standard_normal((l0 + 1, 7)))
    g00 = np.array([0.2, 1.3, -0.7])
    f = rng.standard_normal((l0 + 1, nx, np_))
    Ex = rng.standard_normal(nx)
    return ptab, coef, g00, f, Ex


def test_rhs_transpose(lib):
    l0, np_, nx = 3, 24, 7
    ptab, coef, g00, f, Ex = _rhs_case(l0, np_, nx)
    rng = np.random.default_rng(9)

    def F(f_, E_):
        sf = np.zeros_like(f_)
        sE = np.zeros(nx)
        lib.ac_rhs(np_, nx, l0, P(ptab), P(coef), P(g00), P(np.ascontiguousarray(f_)), P(np.ascontiguousarray(E_)),
                   P(sf), P(sE))
        return sf, sE
    cf = rng.standard_normal(f.shape)
    cE = rng.standard_normal(nx)
    df = rng.standard_normal(f.shape)
    dE = rng.standard_normal(nx)
    eps = 1e-3
    s1f, s1E = F(f + eps * df, Ex + eps * dE)
    s0f, s0E = F(f - eps * df, Ex - eps * dE)
    lhs = (np.sum(cf * (s1f - s0f)) + np.dot(cE, s1E - s0E)) / (2 * eps)
    # the transpose knows nothing of masked outputs: zero their cotangents as the kernels receive them
    lf = np.zeros_like(f)
    lE = np.zeros(nx)
    lib.ac_vjp(np_, nx, l0, P(ptab), P(coef), P(g00), P(f), P(Ex), P(cf), P(cE), P(lf), P(lE))
    rhs = np.sum(lf * df) + np.dot(lE, dE)
    assert abs(lhs - rhs) <= 1e-10 * (abs(lhs) + abs(rhs)), (lhs, rhs)
