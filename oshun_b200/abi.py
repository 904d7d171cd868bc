"""ctypes binding of liboshun_b200.so (the C ABI in include/oshun_b200.h).

Used by the tests and bench.py to drive the CUDA path exactly as a foreign
caller would.  There is no fallback: if the library is missing or no B200 is
present, construction raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# OSHUN_B200_LIB points at another build of the library (default: the in-tree one)
LIB_PATH = os.environ.get("OSHUN_B200_LIB") or os.path.join(HERE, "liboshun_b200.so")

OSHUN_FP64 = 0
OSHUN_FP32_SPLIT = 1
OSHUN_FLAG_FIX_YADV_CHAIN = 0x1
OSHUN_FLAG_IMPLICIT_EE = 0x2      # opt-in backward-Euler f00 e-e step (not a reference scheme)

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_UNSUPPORTED", 3: "ERR_CUDA", 4: "ERR_NONREAL",
          5: "ERR_NUMERIC", 6: "ERR_NO_DEVICE"}

EXPORTED = [
    "oshun_create", "oshun_destroy", "oshun_set_stream", "oshun_synchronize", "oshun_upload",
    "oshun_download", "oshun_rhs", "oshun_rk4_step", "oshun_collide_ee", "oshun_collide_f1",
    "oshun_collide_flm", "oshun_step", "oshun_time", "oshun_status_flags", "oshun_device_state",
    "oshun_plane_index", "oshun_last_error", "oshun_abi_version", "oshun_collide_flm_noalloc",
    "oshun_batch_create", "oshun_batch_destroy", "oshun_batch_set_stream", "oshun_batch_size", "oshun_batch_problem",
    "oshun_batch_upload", "oshun_batch_download", "oshun_batch_step", "oshun_batch_status",
    "oshun_batch_set_tiles", "oshun_batch_get_tiles", "oshun_batch_autotune",
    "oshun_adjoint_create", "oshun_adjoint_destroy", "oshun_adjoint_set_stream", "oshun_adjoint_state_size",
    "oshun_adjoint_forward", "oshun_adjoint_vjp", "oshun_debug_inject_stage_timeout", "oshun_get_config",
    "oshun_moments", "oshun_restart_bytes", "oshun_restart_pack", "oshun_restart_unpack", "oshun_restart_write",
    "oshun_restart_read", "oshun_rk2_imp_step", "oshun_plane_profile",
    "oshun_set_x_boundary", "oshun_halo_bytes", "oshun_halo_pack", "oshun_halo_unpack", "oshun_halo_mirror_side",
    "oshun_step_stage",
]
OSHUN_XB_PERIODIC, OSHUN_XB_MIRROR, OSHUN_XB_HALO = 0, 1, 2


class OshunCfg(ctypes.Structure):
    _fields_ = [
        ("l0", ctypes.c_int), ("m0", ctypes.c_int),
        ("nump", ctypes.c_int), ("numx", ctypes.c_int), ("numy", ctypes.c_int),
        ("pmin", ctypes.c_double), ("pmax", ctypes.c_double),
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
        ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
        ("dt", ctypes.c_double), ("t0", ctypes.c_double), ("small_dt", ctypes.c_double),
        ("NB_algorithms", ctypes.c_int), ("if_tridiagonal", ctypes.c_int), ("if_implicit1D", ctypes.c_int),
        ("density_np", ctypes.c_double), ("Zeta", ctypes.c_double),
        ("precision", ctypes.c_int), ("flags", ctypes.c_int),
    ]


class OshunError(RuntimeError):
    def __init__(self, code: int, what: str, msg: str):
        super().__init__(f"{what}: {STATUS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the library once; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built (python -m oshun_b200.build)")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    lib.oshun_create.argtypes = [ctypes.POINTER(OshunCfg), ctypes.POINTER(vp)]
    lib.oshun_destroy.argtypes = [vp]
    lib.oshun_set_stream.argtypes = [vp, vp]
    lib.oshun_synchronize.argtypes = [vp]
    lib.oshun_upload.argtypes = [vp, vp, vp]
    lib.oshun_download.argtypes = [vp, vp, vp]
    lib.oshun_rhs.argtypes = [vp, vp, vp]
    lib.oshun_rk4_step.argtypes = [vp]
    lib.oshun_collide_ee.argtypes = [vp, ctypes.c_double]
    lib.oshun_collide_f1.argtypes = [vp, ctypes.c_double]
    lib.oshun_collide_flm.argtypes = [vp, ctypes.c_double]
    lib.oshun_step.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.oshun_time.argtypes = [vp, dp]
    lib.oshun_status_flags.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]
    lib.oshun_device_state.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                       ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    lib.oshun_plane_index.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.oshun_debug_inject_stage_timeout.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    lib.oshun_get_config.argtypes = [vp, ctypes.POINTER(OshunCfg)]
    lib.oshun_rk2_imp_step.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.oshun_set_x_boundary.argtypes = [vp, ctypes.c_int]
    lib.oshun_halo_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.oshun_halo_pack.argtypes = [vp, vp, vp]
    lib.oshun_halo_unpack.argtypes = [vp, vp, vp]
    lib.oshun_step_stage.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.oshun_halo_mirror_side.argtypes = [vp, ctypes.c_int]
    lib.oshun_plane_profile.argtypes = [vp, ctypes.POINTER(vp)]
    lib.oshun_moments.argtypes = [vp, vp]
    lib.oshun_restart_bytes.argtypes = [ctypes.POINTER(OshunCfg), ctypes.c_int]
    lib.oshun_restart_bytes.restype = ctypes.c_longlong
    lib.oshun_restart_pack.argtypes = [ctypes.POINTER(OshunCfg), ctypes.c_int, vp, vp, vp]
    lib.oshun_restart_unpack.argtypes = [ctypes.POINTER(OshunCfg), ctypes.c_int, vp, vp, vp]
    lib.oshun_restart_write.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.oshun_restart_read.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.oshun_collide_flm_noalloc.argtypes = [ctypes.POINTER(OshunCfg), vp, vp, ctypes.c_double, vp,
                                              ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
    ip = ctypes.POINTER(ctypes.c_int)
    if not hasattr(lib, "oshun_batch_create"):   # a build without the batch entry points
        lib.oshun_last_error.restype = ctypes.c_char_p
        lib.oshun_abi_version.restype = ctypes.c_int
        _lib = lib
        return lib
    lib.oshun_batch_create.argtypes = [ctypes.POINTER(OshunCfg), ctypes.c_int, ip, ctypes.POINTER(vp)]
    lib.oshun_batch_destroy.argtypes = [vp]
    lib.oshun_batch_size.argtypes = [vp, ip]
    lib.oshun_batch_set_stream.argtypes = [vp, vp]
    lib.oshun_batch_problem.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
    lib.oshun_batch_upload.argtypes = [vp, ctypes.c_int, vp, vp]
    lib.oshun_batch_download.argtypes = [vp, ctypes.c_int, vp, vp]
    lib.oshun_batch_step.argtypes = [vp, ctypes.c_int]
    lib.oshun_batch_status.argtypes = [vp, ip]
    lib.oshun_batch_set_tiles.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.oshun_batch_get_tiles.argtypes = [vp, ip, ip]
    lib.oshun_batch_autotune.argtypes = [vp, ctypes.c_int, ip, ip, dp]
    if hasattr(lib, "oshun_adjoint_create"):
        d = ctypes.c_double
        lib.oshun_adjoint_create.argtypes = [ctypes.POINTER(OshunCfg), ctypes.POINTER(vp)]
        lib.oshun_adjoint_destroy.argtypes = [vp]
        lib.oshun_adjoint_set_stream.argtypes = [vp, vp]
        lib.oshun_adjoint_state_size.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        lib.oshun_adjoint_forward.argtypes = [vp, vp, vp, ctypes.c_int, d, d, d]
        lib.oshun_adjoint_vjp.argtypes = [vp, vp, vp, vp, ctypes.c_int, d, d, d]
    lib.oshun_last_error.restype = ctypes.c_char_p
    lib.oshun_abi_version.restype = ctypes.c_int
    _lib = lib
    return lib


def make_cfg(**kw) -> OshunCfg:
    c = OshunCfg()
    defaults = dict(t0=0.0, precision=OSHUN_FP64, flags=0, NB_algorithms=4, if_tridiagonal=1,
                    if_implicit1D=1, density_np=1e21, Zeta=1.0, ymin=0.0, ymax=1.0, small_dt=1.0)
    defaults.update(kw)
    for name, _ in OshunCfg._fields_:
        if name not in defaults:
            raise KeyError(f"oshun_cfg field {name} missing")
        setattr(c, name, defaults[name])
    return c


class Handle:
    """One oshun_handle: the device state of one run and its operators."""

    def __init__(self, **cfg):
        self.lib = load()
        self.cfg = make_cfg(**cfg)
        self._h = ctypes.c_void_p()
        self._check(self.lib.oshun_create(ctypes.byref(self.cfg), ctypes.byref(self._h)), "oshun_create")
        c = self.cfg
        self.nh = ((c.m0 + 1) * (2 * c.l0 - c.m0 + 2)) // 2
        self.fshape = (self.nh, c.numy, c.numx, c.nump)
        self.fldshape = (6, c.numy, c.numx)

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            raise OshunError(rc, what, self.lib.oshun_last_error().decode())

    def close(self) -> None:
        if self._h:
            self.lib.oshun_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _ptr(a: np.ndarray) -> ctypes.c_void_p:
        return ctypes.c_void_p(a.ctypes.data)

    def upload(self, f: np.ndarray, fields: np.ndarray) -> None:
        f = np.ascontiguousarray(f, np.complex128)
        fields = np.ascontiguousarray(fields, np.complex128)
        assert f.shape == self.fshape and fields.shape == self.fldshape
        self._check(self.lib.oshun_upload(self._h, self._ptr(f), self._ptr(fields)), "oshun_upload")

    def upload_ptr(self, f_ptr: int, fields_ptr: int) -> None:
        self._check(self.lib.oshun_upload(self._h, ctypes.c_void_p(f_ptr), ctypes.c_void_p(fields_ptr)),
                    "oshun_upload")

    def download(self):
        f = np.empty(self.fshape, np.complex128)
        fields = np.empty(self.fldshape, np.complex128)
        self._check(self.lib.oshun_download(self._h, self._ptr(f), self._ptr(fields)), "oshun_download")
        return f, fields

    def download_ptr(self, f_ptr: int, fields_ptr: int) -> None:
        self._check(self.lib.oshun_download(self._h, ctypes.c_void_p(f_ptr), ctypes.c_void_p(fields_ptr)),
                    "oshun_download")

    def rhs(self):
        f = np.empty(self.fshape, np.complex128)
        fields = np.empty(self.fldshape, np.complex128)
        self._check(self.lib.oshun_rhs(self._h, self._ptr(f), self._ptr(fields)), "oshun_rhs")
        return f, fields

    def rk4_step(self) -> None:
        self._check(self.lib.oshun_rk4_step(self._h), "oshun_rk4_step")

    def collide_ee(self, t_new: float) -> None:
        self._check(self.lib.oshun_collide_ee(self._h, t_new), "oshun_collide_ee")

    def collide_f1(self, t_new: float) -> None:
        self._check(self.lib.oshun_collide_f1(self._h, t_new), "oshun_collide_f1")

    def collide_flm(self, t_new: float) -> None:
        self._check(self.lib.oshun_collide_flm(self._h, t_new), "oshun_collide_flm")

    def step(self, nsteps: int, collisions: bool = True) -> None:
        self._check(self.lib.oshun_step(self._h, nsteps, 1 if collisions else 0), "oshun_step")

    def rk2_imp_step(self, nsteps: int, mask: int = 63) -> None:
        """nsteps of the implicit-E small step (mask bits as oshun_rk2_imp_step)."""
        self._check(self.lib.oshun_rk2_imp_step(self._h, nsteps, mask), "oshun_rk2_imp_step")

    def plane_index(self, l: int, m: int) -> int:
        """Plane of Re f_lm (l >= 1; Im follows), -1 for f00."""
        q = ctypes.c_int()
        self._check(self.lib.oshun_plane_index(self._h, l, m, ctypes.byref(q)), "oshun_plane_index")
        return q.value

    def set_x_boundary(self, mode: int) -> None:
        """OSHUN_XB_PERIODIC, OSHUN_XB_MIRROR or OSHUN_XB_HALO (an x slab)."""
        self._check(self.lib.oshun_set_x_boundary(self._h, int(mode)), "oshun_set_x_boundary")

    def halo_bytes(self) -> int:
        n = ctypes.c_longlong()
        self._check(self.lib.oshun_halo_bytes(self._h, ctypes.byref(n)), "oshun_halo_bytes")
        return n.value

    def halo_pack(self, left_edge: int, right_edge: int) -> None:
        """The next stage's edge columns into two device buffers (pointers)."""
        self._check(self.lib.oshun_halo_pack(self._h, left_edge, right_edge), "oshun_halo_pack")

    def halo_unpack(self, from_left: int, from_right: int) -> None:
        """The neighbours' edge columns (device pointers) into the halo."""
        self._check(self.lib.oshun_halo_unpack(self._h, from_left, from_right), "oshun_halo_unpack")

    def halo_mirror_side(self, side: int) -> None:
        """Side 0 (left) or 1 (right) of the halo as a mirrored boundary."""
        self._check(self.lib.oshun_halo_mirror_side(self._h, int(side)), "oshun_halo_mirror_side")

    def step_stage(self, k: int, collisions: bool = True) -> None:
        """RK4 stage k (1..4) of the small step; stage 4 also collides."""
        self._check(self.lib.oshun_step_stage(self._h, int(k), int(bool(collisions))), "oshun_step_stage")

    def synchronize(self) -> None:
        self._check(self.lib.oshun_synchronize(self._h), "oshun_synchronize")

    def set_stream(self, stream_ptr: int | None) -> None:
        self._check(self.lib.oshun_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)), "oshun_set_stream")

    @property
    def time(self) -> float:
        t = ctypes.c_double()
        self._check(self.lib.oshun_time(self._h, ctypes.byref(t)), "oshun_time")
        return t.value

    def inject_stage_timeout(self, withhold_copy: int, wait_seconds: float) -> None:
        """Fault injection for tests: the next rk4_step's stage launches stop
        one copy short and their waits give up after wait_seconds."""
        self._check(self.lib.oshun_debug_inject_stage_timeout(self._h, withhold_copy, wait_seconds),
                    "oshun_debug_inject_stage_timeout")

    MOMENTS = ("N", "Vx", "Vy", "VxVx", "VyVy", "VzVz", "VxVy", "VxVz", "VyVz", "Vsq", "T_eV", "P_Mbar", "ND",
               "Nu", "Qx", "Kx", "Qy", "Ky")

    def moments(self) -> np.ndarray:
        """float32 [18][numy][numx]: Parallel_Output::nonrelativistic_moments
        of the current state, computed on the device (order: MOMENTS)."""
        out = np.empty((len(self.MOMENTS), self.cfg.numy, self.cfg.numx), np.float32)
        self._check(self.lib.oshun_moments(self._h, self._ptr(out)), "oshun_moments")
        return out

    def restart_write(self, prefix: str, rank: int, re_step: int, guard_cells: int = 4) -> None:
        self._check(self.lib.oshun_restart_write(self._h, prefix.encode(), rank, re_step, guard_cells),
                    "oshun_restart_write")

    def restart_read(self, prefix: str, rank: int, re_step: int, guard_cells: int = 4) -> None:
        self._check(self.lib.oshun_restart_read(self._h, prefix.encode(), rank, re_step, guard_cells),
                    "oshun_restart_read")

    def status_flags(self):
        fl = ctypes.c_int()
        cnt = ctypes.c_longlong()
        self._check(self.lib.oshun_status_flags(self._h, ctypes.byref(fl), ctypes.byref(cnt)), "oshun_status_flags")
        return fl.value, cnt.value

    def device_state(self):
        f00, pl, fl = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        pb, fb = ctypes.c_size_t(), ctypes.c_size_t()
        self._check(self.lib.oshun_device_state(self._h, ctypes.byref(f00), ctypes.byref(pl), ctypes.byref(fl),
                                                ctypes.byref(pb), ctypes.byref(fb)), "oshun_device_state")
        return f00.value, pl.value, fl.value, pb.value, fb.value


def restart_pack(cfg: dict, f: np.ndarray, fields: np.ndarray, guard_cells: int = 4) -> bytes:
    """The reference's restart-file image of a host state (no device needed)."""
    lib = load()
    c = make_cfg(**cfg)
    n = lib.oshun_restart_bytes(ctypes.byref(c), guard_cells)
    if n < 0:
        raise OshunError(1, "oshun_restart_bytes", lib.oshun_last_error().decode())
    img = np.empty(n // 8, np.float64)
    f = np.ascontiguousarray(f, np.complex128)
    fields = np.ascontiguousarray(fields, np.complex128)
    rc = lib.oshun_restart_pack(ctypes.byref(c), guard_cells, f.ctypes.data, fields.ctypes.data, img.ctypes.data)
    if rc:
        raise OshunError(rc, "oshun_restart_pack", lib.oshun_last_error().decode())
    return img.tobytes()


def restart_unpack(cfg: dict, image: bytes, guard_cells: int = 4):
    """Interior state (f, fields) of a restart-file image."""
    lib = load()
    c = make_cfg(**cfg)
    n = lib.oshun_restart_bytes(ctypes.byref(c), guard_cells)
    if n != len(image):
        raise OshunError(1, "oshun_restart_unpack", f"image holds {len(image)} bytes, the configuration {n}")
    nh = ((c.m0 + 1) * (2 * c.l0 - c.m0 + 2)) // 2
    f = np.empty((nh, c.numy, c.numx, c.nump), np.complex128)
    fields = np.empty((6, c.numy, c.numx), np.complex128)
    img = np.frombuffer(image, np.float64)
    rc = lib.oshun_restart_unpack(ctypes.byref(c), guard_cells, img.ctypes.data, f.ctypes.data, fields.ctypes.data)
    if rc:
        raise OshunError(rc, "oshun_restart_unpack", lib.oshun_last_error().decode())
    return f, fields


class Batch:
    """One oshun_batch: independent problems advanced together, one captured
    graph per step (see include/oshun_b200.h)."""

    def __init__(self, cfgs, collide=None):
        self.lib = load()
        self.cfgs = [make_cfg(**c) for c in cfgs]
        n = len(self.cfgs)
        arr = (OshunCfg * n)(*self.cfgs)
        col = None
        if collide is not None:
            col = (ctypes.c_int * n)(*[int(bool(x)) for x in collide])
        self._b = ctypes.c_void_p()
        self._check(self.lib.oshun_batch_create(arr, n, col, ctypes.byref(self._b)), "oshun_batch_create")
        self.n = n
        self.shapes = []
        for c in self.cfgs:
            nh = ((c.m0 + 1) * (2 * c.l0 - c.m0 + 2)) // 2
            self.shapes.append(((nh, c.numy, c.numx, c.nump), (6, c.numy, c.numx)))

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            raise OshunError(rc, what, self.lib.oshun_last_error().decode())

    def close(self) -> None:
        if self._b:
            self.lib.oshun_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, i: int, f: np.ndarray, fields: np.ndarray) -> None:
        f = np.ascontiguousarray(f, np.complex128)
        fields = np.ascontiguousarray(fields, np.complex128)
        assert f.shape == self.shapes[i][0] and fields.shape == self.shapes[i][1]
        self._check(self.lib.oshun_batch_upload(self._b, i, f.ctypes.data, fields.ctypes.data), "oshun_batch_upload")

    def download(self, i: int):
        f = np.empty(self.shapes[i][0], np.complex128)
        fields = np.empty(self.shapes[i][1], np.complex128)
        self._check(self.lib.oshun_batch_download(self._b, i, f.ctypes.data, fields.ctypes.data),
                    "oshun_batch_download")
        return f, fields

    def step(self, nsteps: int = 1) -> None:
        self._check(self.lib.oshun_batch_step(self._b, nsteps), "oshun_batch_step")

    def set_stream(self, stream_ptr: int) -> None:
        """Run on this cudaStream_t (an integer handle, 0 = the batch's own stream)."""
        self._check(self.lib.oshun_batch_set_stream(self._b, ctypes.c_void_p(stream_ptr or None)),
                    "oshun_batch_set_stream")

    def status(self) -> int:
        f = ctypes.c_int()
        self._check(self.lib.oshun_batch_status(self._b, ctypes.byref(f)), "oshun_batch_status")
        return f.value

    def set_tiles(self, stage_threads: int, tile_cells: int) -> None:
        self._check(self.lib.oshun_batch_set_tiles(self._b, stage_threads, tile_cells), "oshun_batch_set_tiles")

    def tiles(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.oshun_batch_get_tiles(self._b, ctypes.byref(a), ctypes.byref(b)), "oshun_batch_get_tiles")
        return a.value, b.value

    def autotune(self, steps: int = 2):
        a, b, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.oshun_batch_autotune(self._b, steps, ctypes.byref(a), ctypes.byref(b), ctypes.byref(ms)),
                    "oshun_batch_autotune")
        return a.value, b.value, ms.value

