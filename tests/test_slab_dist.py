"""oshun_b200.slab's neighbour exchange on the CPU: 2 and 3 gloo ranks
(RANK, WORLD_SIZE, MASTER_ADDR = 127.0.0.1) run XSlab's real exchange code
against a stand-in handle whose halo_pack writes rank-tagged edge columns
into the send buffers and whose halo_unpack records what arrived.  Every
rank must receive its left neighbour's right edge and its right
neighbour's left edge (periodic in x), the end ranks of a mirrored split
mirror their outer sides, and the four stages run in order after each
exchange.  The slab configuration keeps the whole grid's dx bit for bit."""
import json
import os
import sys

import pytest

from tests.test_bench_dist import _launch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, os, sys
sys.path.insert(0, {root!r})
import torch, torch.distributed as dist
dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
rank, ws = dist.get_rank(), dist.get_world_size()
from oshun_b200.slab import XSlab
N = 64

class FakeHandle:
    def __init__(self, rank):
        self.rank, self.log = rank, []
    def halo_pack(self, pl, pr):
        ctypes.memmove(pl, bytes([10 * self.rank + 1]) * N, N)
        ctypes.memmove(pr, bytes([10 * self.rank + 2]) * N, N)
        self.log.append("pack")
    def halo_unpack(self, fl, fr):
        a = ctypes.string_at(fl, N)
        b = ctypes.string_at(fr, N)
        assert len(set(a)) == 1 and len(set(b)) == 1
        self.log.append(("unpack", a[0], b[0]))
    def halo_mirror_side(self, side):
        self.log.append(("mirror", side))
    def step_stage(self, k, col):
        self.log.append(("stage", k))

mirror = {mirror}
s = XSlab.__new__(XSlab)
s.rank, s.world, s.group, s.mirror = rank, ws, None, mirror
s.h = FakeHandle(rank)
s.send_l, s.send_r, s.recv_l, s.recv_r = (torch.zeros(N, dtype=torch.uint8) for _ in range(4))
s.step(2)
print(json.dumps(dict(rank=rank, ws=ws, log=s.h.log)), flush=True)
dist.destroy_process_group()
"""


@pytest.mark.parametrize("ws", [2, 3])
@pytest.mark.parametrize("mirror", [False, True])
def test_slab_exchange_neighbours(ws, mirror):
    outs = _launch(CHILD.format(root=ROOT, mirror=mirror), ws=ws)
    recs = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert {r["rank"] for r in recs} == set(range(ws))
    for r in recs:
        rank = r["rank"]
        left, right = (rank - 1) % ws, (rank + 1) % ws
        log = [tuple(e) if isinstance(e, list) else e for e in r["log"]]
        unpacks = [e for e in log if isinstance(e, tuple) and e[0] == "unpack"]
        stages = [e[1] for e in log if isinstance(e, tuple) and e[0] == "stage"]
        assert stages == [1, 2, 3, 4, 1, 2, 3, 4]
        assert len(unpacks) == 8 and log.count("pack") == 8
        for e in unpacks:
            assert e[1] == 10 * left + 2 and e[2] == 10 * right + 1
        mirrors = [e[1] for e in log if isinstance(e, tuple) and e[0] == "mirror"]
        want = ([0] if rank == 0 else []) + ([1] if rank == ws - 1 else [])
        assert mirrors == (want * 8 if mirror else [])
        # every stage runs after its exchange
        for i, e in enumerate(log):
            if isinstance(e, tuple) and e[0] == "stage":
                prev = [x for x in log[:i] if isinstance(x, tuple) and x[0] in ("unpack", "stage")]
                assert prev[-1][0] == "unpack"


def test_slab_cfg_keeps_dx():
    from oshun_b200.slab import slab_cfg
    for nx, xmax, ws in ((12, 2.75, 2), (30, 1.0, 3), (128, 127 * 0.1, 8), (96, 7.3, 4)):
        cfg = dict(numx=nx, xmin=0.0, xmax=xmax)
        dx = (xmax - 0.0) / (nx - 1)
        for r in range(ws):
            c = slab_cfg(cfg, r, ws)
            assert c["numx"] == nx // ws
            assert (c["xmax"] - c["xmin"]) / (c["numx"] - 1) == dx
    with pytest.raises(ValueError):
        slab_cfg(dict(numx=10, xmin=0.0, xmax=1.0), 0, 3)
