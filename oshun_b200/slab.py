"""A grid split over ranks in x (one x slab per rank, one process per GPU):
the reference's x decomposition with its neighbour exchange
(OSHUN-1/def-Parallel.cpp:3040-3129, Parallel_Environment::
Neighbor_Communications) on the C ABI's halo entry points.

    slab = XSlab(cfg, rank, world)          # cfg: the whole grid's configuration
    slab.upload(f_slab, fields_slab)        # this rank's columns of the state
    slab.step(nsteps)                       # RK4 small steps (+ collisions)

Each RK4 stage needs the x-1 neighbour of the slab's first column and the
x+1 neighbour of its last: before every stage each rank packs its two edge
columns (oshun_halo_pack), sends the left one to the left rank and the right
one to the right rank and receives theirs (one batch of point-to-point
operations on the process group: NCCL over NVLink between GPUs), loads them
(oshun_halo_unpack) and runs the stage (oshun_step_stage).  With mirrored x
boundaries (bndX = 1) the first rank's left halo and the last rank's right
halo are the mirror images of their own edge columns (oshun_halo_mirror_side)
instead.  Collisions act per cell and need no exchange.  Every rank takes
the same collective steps in the same order.

The slab's arithmetic is the whole grid's, cell by cell, so a split run is
bit-identical to the single-grid run (tests/test_gpu_xslab.py emulates the
split on one GPU; tests/test_slab_dist.py runs the exchange with gloo ranks).
"""
from __future__ import annotations

import math

from .abi import OSHUN_XB_HALO, Handle


def slab_cfg(cfg: dict, rank: int, world: int) -> dict:
    """This rank's configuration: numx / world columns with the whole grid's dx."""
    nx = cfg["numx"]
    if world < 1 or nx % world != 0 or nx // world < 2:
        raise ValueError("numx must split into world slabs of at least 2 columns")
    nxl = nx // world
    dx = (cfg["xmax"] - cfg["xmin"]) / (nx - 1)
    xmax = dx * (nxl - 1)
    # the handle derives dx = (xmax - xmin) / (numx - 1): match the grid's bit for bit
    for _ in range(64):
        got = xmax / (nxl - 1)
        if got == dx:
            break
        xmax = math.nextafter(xmax, math.inf if got < dx else -math.inf)
    else:
        raise ValueError("no slab axis reproduces the grid's dx")
    return dict(cfg, numx=nxl, xmin=0.0, xmax=xmax)


class XSlab:
    """One rank's slab; `group` is a torch.distributed process group (None:
    the default group; world == 1 runs without any collective)."""

    def __init__(self, cfg: dict, rank: int, world: int, group=None, mirror: bool = False, device=None):
        import torch
        self.rank, self.world, self.group, self.mirror = rank, world, group, mirror
        self.cfg = slab_cfg(cfg, rank, world)
        self.h = Handle(**self.cfg)
        self.h.set_x_boundary(OSHUN_XB_HALO)
        n = self.h.halo_bytes()
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.send_l, self.send_r, self.recv_l, self.recv_r = (
            torch.empty(n, dtype=torch.uint8, device=dev) for _ in range(4))

    def close(self) -> None:
        self.h.close()

    def upload(self, f, fields) -> None:
        self.h.upload(f, fields)

    def download(self):
        return self.h.download()

    def _exchange(self) -> None:
        import torch
        self.h.halo_pack(self.send_l.data_ptr(), self.send_r.data_ptr())
        if self.world == 1:
            self.recv_l.copy_(self.send_r)
            self.recv_r.copy_(self.send_l)
            if self.recv_l.is_cuda:
                torch.cuda.current_stream().synchronize()
        else:
            import torch.distributed as dist
            left, right = (self.rank - 1) % self.world, (self.rank + 1) % self.world
            ops = [dist.P2POp(dist.isend, self.send_r, right, self.group),
                   dist.P2POp(dist.irecv, self.recv_l, left, self.group),
                   dist.P2POp(dist.isend, self.send_l, left, self.group),
                   dist.P2POp(dist.irecv, self.recv_r, right, self.group)]
            for r in dist.batch_isend_irecv(ops):
                r.wait()
            if self.recv_l.is_cuda:
                torch.cuda.current_stream().synchronize()
        self.h.halo_unpack(self.recv_l.data_ptr(), self.recv_r.data_ptr())
        if self.mirror and self.rank == 0:
            self.h.halo_mirror_side(0)
        if self.mirror and self.rank == self.world - 1:
            self.h.halo_mirror_side(1)

    def step(self, nsteps: int = 1, collisions: bool = True) -> None:
        for _ in range(nsteps):
            for k in (1, 2, 3, 4):
                self._exchange()
                self.h.step_stage(k, collisions)
