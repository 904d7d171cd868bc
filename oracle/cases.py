"""Case files, seeded inputs and the CPU checkers — TEST INFRASTRUCTURE ONLY.

Imported by tests/, by ``__graft_entry__.smoke()`` and by ``bench.py``'s
CPU-baseline leg, and only there, as the checker.  The product path
(``oshun_b200``) never imports this module.

* ``Deck``            the case header shared with oracle/ref_harness/harness.cpp
                      and oracle/oshun_oracle.c (the reference's input-deck
                      fields on the hot path, OSHUN-1/decl-input.h:59-138).
* ``write_case`` / ``read_case``   the binary case format.
* ``seeded_state``    Maxwellian f00 (OSHUN-1/def-Setup.cpp:500-533) with
                      seeded perturbations of the other harmonics and fields.
* ``Oracle``          ctypes binding of liboshun_oracle.so (the C restatement).
* ``run_reference``   runs the reference's own code (oracle/_ref/oshun_ref).
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "oshun_ref")
ORACLE_SO = os.path.join(HERE, "liboshun_oracle.so")

INT_FIELDS = ("l0", "m0", "nump", "numx", "numy", "NB_algorithms", "if_tridiagonal", "if_implicit1D")
DBL_FIELDS = ("pmin", "pmax", "xmin", "xmax", "ymin", "ymax", "dt", "small_dt", "density_np", "Zeta")


@dataclasses.dataclass
class Deck:
    l0: int
    m0: int
    nump: int
    numx: int
    numy: int = 1
    NB_algorithms: int = 4
    if_tridiagonal: int = 1
    if_implicit1D: int = 1
    pmin: float = 0.0
    pmax: float = 0.4
    xmin: float = 0.0
    xmax: float = 1.0
    ymin: float = 0.0
    ymax: float = 1.0
    dt: float = 0.05
    small_dt: float = 0.05
    density_np: float = 1.0e21
    Zeta: float = 1.0

    def __post_init__(self):
        if self.pmin == 0.0:
            # the reference decks set pmin = pmax / (2 nump) (OSHUN-1/def-Input.cpp:79)
            self.pmin = self.pmax / (2.0 * self.nump)

    @property
    def nh(self) -> int:
        return ((self.m0 + 1) * (2 * self.l0 - self.m0 + 2)) // 2

    @property
    def cells(self) -> int:
        return self.numx * self.numy

    def ind(self, l: int, m: int) -> int:
        """ind(l,m) of OSHUN-1/def-State.cpp:420-427."""
        if l < self.m0 + 1:
            return (l * (l + 1)) // 2 + m
        return l * (self.m0 + 1) - (self.m0 * (self.m0 + 1)) // 2 + m

    def harmonics(self):
        for l in range(self.l0 + 1):
            for m in range(min(l, self.m0) + 1):
                yield l, m

    def pr(self) -> np.ndarray:
        i = np.arange(self.nump, dtype=np.float64)
        return i * ((self.pmax - self.pmin) / (self.nump - 1)) + self.pmin

    def dx_periodic(self) -> float:
        """Cell width; the periodic domain holds numx cells."""
        return (self.xmax - self.xmin) / (self.numx - 1)

    def pack_header(self) -> bytes:
        return (b"OSHC" + struct.pack("<i", 1)
                + struct.pack("<8i", *[int(getattr(self, k)) for k in INT_FIELDS])
                + struct.pack("<10d", *[float(getattr(self, k)) for k in DBL_FIELDS]))

    def replace(self, **kw) -> "Deck":
        d = dataclasses.replace(self, **kw)
        if "pmax" in kw or "nump" in kw:
            if "pmin" not in kw:
                d.pmin = d.pmax / (2.0 * d.nump)
        return d


class State:
    """Complex state in the case layout: f[Nh][ny][nx][np], fields[6][ny][nx]."""

    def __init__(self, deck: Deck, f: np.ndarray | None = None, fields: np.ndarray | None = None):
        self.deck = deck
        shp = (deck.nh, deck.numy, deck.numx, deck.nump)
        self.f = np.zeros(shp, np.complex128) if f is None else np.ascontiguousarray(f, np.complex128)
        self.fields = (np.zeros((6, deck.numy, deck.numx), np.complex128) if fields is None
                       else np.ascontiguousarray(fields, np.complex128))
        assert self.f.shape == shp and self.fields.shape == (6, deck.numy, deck.numx)

    def flat(self) -> np.ndarray:
        return np.concatenate([self.f.ravel(), self.fields.ravel()]).view(np.float64)

    @classmethod
    def from_flat(cls, deck: Deck, buf: np.ndarray) -> "State":
        c = np.ascontiguousarray(buf, np.float64).view(np.complex128)
        n = deck.nh * deck.cells * deck.nump
        f = c[:n].reshape(deck.nh, deck.numy, deck.numx, deck.nump)
        fields = c[n:].reshape(6, deck.numy, deck.numx)
        return cls(deck, f.copy(), fields.copy())

    def copy(self) -> "State":
        return State(self.deck, self.f.copy(), self.fields.copy())

    def harmonic(self, l: int, m: int) -> np.ndarray:
        return self.f[self.deck.ind(l, m)]


def write_case(path: str, st: State) -> None:
    with open(path, "wb") as fh:
        fh.write(st.deck.pack_header())
        fh.write(st.flat().tobytes())


def read_case(path: str) -> State:
    with open(path, "rb") as fh:
        raw = fh.read()
    assert raw[:4] == b"OSHC" and struct.unpack("<i", raw[4:8])[0] == 1
    iv = struct.unpack("<8i", raw[8:40])
    dv = struct.unpack("<10d", raw[40:120])
    kw = dict(zip(INT_FIELDS, iv))
    kw.update(zip(DBL_FIELDS, dv))
    deck = Deck(**kw)
    return State.from_flat(deck, np.frombuffer(raw[120:], np.float64))


# ----------------------------------------------------------------------------
# seeded inputs
# ----------------------------------------------------------------------------

def maxwellian(p: np.ndarray, pt: np.ndarray) -> np.ndarray:
    """exp(-p^2/2pt^2) / ((2 pi)^{3/2} pt^3), Setup_Y::Gaussian_p
    (OSHUN-1/def-Setup.cpp:500-533)."""
    return np.exp(-(p * p) / (2.0 * pt * pt)) / (np.sqrt(2.0 * np.pi) * 2.0 * np.pi * pt ** 3)


def seeded_state(deck: Deck, seed: int = 0, vth: float = 0.05, amp: float = 1e-2,
                 fields: bool = True, aniso: bool = True) -> State:
    """Maxwellian f00 with a seeded density and temperature ripple, seeded
    smooth higher harmonics (f_lm ~ amp * (p/vth)^l * Maxwellian) and, when
    ``fields``, seeded E and B.  m = 0 harmonics and the fields are real, as
    every reference operator keeps them."""
    rng = np.random.default_rng(seed)
    p = deck.pr()
    ny, nx = deck.numy, deck.numx
    kx = 2.0 * np.pi * np.arange(nx) / nx
    ky = 2.0 * np.pi * np.arange(ny) / ny
    X, Yy = np.meshgrid(kx, ky)                      # [ny][nx]
    ph = rng.uniform(0, 2 * np.pi, 4)
    dens = 1.0 + amp * np.cos(X + ph[0]) * (1.0 + 0.5 * np.cos(Yy + ph[1]))
    temp = vth * (1.0 + amp * np.sin(X + ph[2]) + 0.5 * amp * np.cos(Yy + ph[3]))
    st = State(deck)
    st.f[deck.ind(0, 0)] = dens[..., None] * maxwellian(p[None, None, :], temp[..., None])
    f00 = st.f[deck.ind(0, 0)].real.copy()
    if aniso:
        for (l, m) in deck.harmonics():
            if l == 0:
                continue
            a = rng.standard_normal((2, 3))
            sx = (a[0, 0] * np.cos(X) + a[0, 1] * np.sin(X) + a[0, 2] * np.cos(Yy + X))
            sy = (a[1, 0] * np.sin(Yy) + a[1, 1] * np.cos(2 * X) + a[1, 2])
            shape = (p / vth) ** min(l, 3) * (1.0 + 0.3 * np.sin(p / vth + l))
            re = amp * sx[..., None] * shape[None, None, :] * f00
            if m == 0:
                st.f[deck.ind(l, m)] = re
            else:
                im = amp * sy[..., None] * shape[None, None, :] * f00
                st.f[deck.ind(l, m)] = re + 1j * im
    if fields:
        for i in range(6):
            a = rng.standard_normal(3)
            scale = 1e-3 if i < 3 else 5e-4
            st.fields[i] = scale * (a[0] * np.cos(X + a[1]) + a[2] * np.sin(Yy + 0.3 * X))
    return st


def landau_state(deck: Deck, vth: float = 0.05, alpha: float = 1e-3, kmode: int = 1) -> State:
    """1D Landau case: n(x) = 1 + alpha cos(k x), Maxwellian f00, E_x from
    Gauss's law dE/dx = -(n - 1) (electron charge -1, fixed neutralising ions,
    units of the reference: x in c/w_p)."""
    st = State(deck)
    p = deck.pr()
    L = deck.dx_periodic() * deck.numx
    x = np.arange(deck.numx) * deck.dx_periodic()
    k = 2.0 * np.pi * kmode / L
    n = 1.0 + alpha * np.cos(k * x)
    st.f[deck.ind(0, 0), 0] = n[:, None] * maxwellian(p[None, :], np.full(1, vth)[:, None])
    st.fields[0, 0] = -alpha / k * np.sin(k * x)
    return st


# ----------------------------------------------------------------------------
# checkers
# ----------------------------------------------------------------------------

class _OoDeck(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_int) for k in INT_FIELDS] + [(k, ctypes.c_double) for k in DBL_FIELDS])


class Oracle:
    """The C restatement (liboshun_oracle.so)."""

    def __init__(self, path: str = ORACLE_SO):
        self.lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        self.lib.oo_rhs.argtypes = [ctypes.POINTER(_OoDeck), dp, dp]
        self.lib.oo_steps.argtypes = [ctypes.POINTER(_OoDeck), dp, ctypes.c_int, ctypes.c_int]
        self.lib.oo_set_yadv_chain.argtypes = [ctypes.c_int]
        self.lib.oo_set_ee_implicit.argtypes = [ctypes.c_int]
        self.lib.oo_set_mirror_x.argtypes = [ctypes.c_int]
        self.lib.oo_nondominant_count.restype = ctypes.c_long

    @staticmethod
    def _deck(d: Deck) -> _OoDeck:
        return _OoDeck(*[getattr(d, k) for k in INT_FIELDS + DBL_FIELDS])

    def rhs(self, st: State) -> State:
        buf = st.flat().copy()
        out = np.zeros_like(buf)
        dk = self._deck(st.deck)
        dp = ctypes.POINTER(ctypes.c_double)
        rc = self.lib.oo_rhs(ctypes.byref(dk), buf.ctypes.data_as(dp), out.ctypes.data_as(dp))
        assert rc == 0
        return State.from_flat(st.deck, out)

    def steps(self, st: State, nsteps: int, mask: int = 15) -> State:
        buf = st.flat().copy()
        dk = self._deck(st.deck)
        rc = self.lib.oo_steps(ctypes.byref(dk), buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               nsteps, mask)
        assert rc == 0
        return State.from_flat(st.deck, buf)

    def set_yadv_chain(self, keep: bool) -> None:
        self.lib.oo_set_yadv_chain(1 if keep else 0)

    def set_ee_implicit(self, sweeps: int) -> None:
        """0: the reference's explicit e-e substeps; > 0: the opt-in
        backward-Euler e-e step with that many Picard sweeps."""
        self.lib.oo_set_ee_implicit(int(sweeps))

    def set_mirror_x(self, on: bool) -> None:
        """mirrored (True) or periodic (False, default) x boundaries"""
        self.lib.oo_set_mirror_x(1 if on else 0)

    def nondominant(self) -> int:
        return int(self.lib.oo_nondominant_count())


def reference_available() -> bool:
    return os.path.exists(REF_BIN)


def run_reference(st: State, ops, timeout: float = 600.0, time_it: bool = False):
    """Run the reference's own code on ``st``; returns the output state (and
    the step-loop wall time when ``time_it``)."""
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.case"), os.path.join(td, "out.case")
        write_case(fin, st)
        args = [REF_BIN, fin, fout] + list(ops) + (["time"] if time_it else [])
        r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference failed ({r.returncode}): {r.stderr.strip()}")
        out = read_case(fout)
        if time_it:
            t = float(r.stdout.strip().split("elapsed_s=")[-1])
            return out, t
        return out


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Relative L2 error of a against the reference b (absolute if b == 0)."""
    nb = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return float(d / nb) if nb > 0 else float(d)
