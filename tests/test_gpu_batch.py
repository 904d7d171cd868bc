"""Batches of independent problems (oshun_batch_*): one captured graph per
step, persistent batched stage launches, batched collision launches.

* every problem of a mixed batch (1D and 2D, l0, m0, nump, numx and dt all
  different) ends bit-identical to the same problem stepped alone through
  oshun_step, in FP64 and in the FP32/FP64-split form, with and without its
  collision step, and for several stage tilings (the tiles change the work
  split, not the arithmetic);
* the FP64 batch against the oracle: relative L2 <= 1e-12;
* the autotuner leaves the state and the clocks as they were;
* the uneven 512-problem configuration (FP32 bulk) at full size: sampled
  problems bit-identical to solo runs and within 1e-6 of the FP64 oracle.
"""
import numpy as np
import pytest

from oracle.cases import Deck, State, seeded_state
from tests.gpu_util import cfg_of, worst_rel

pytestmark = pytest.mark.gpu


def _mixed(precision):
    decks = [
        Deck(l0=3, m0=0, nump=32, numx=40, dt=0.02, small_dt=0.01, density_np=1e23, xmax=2.0),
        Deck(l0=8, m0=0, nump=64, numx=24, dt=0.05, density_np=5e22, xmax=3.0),
        Deck(l0=4, m0=2, nump=48, numx=8, numy=6, dt=0.02, small_dt=0.05, density_np=1e22, if_implicit1D=0,
             xmax=2.0, ymax=3.0),
        Deck(l0=1, m0=0, nump=128, numx=16, dt=0.04, density_np=1e22, xmax=4.0),
        Deck(l0=6, m0=6, nump=96, numx=6, numy=5, dt=0.02, small_dt=0.05, density_np=1e21, if_implicit1D=0,
             xmax=2.0, ymax=2.0),
        Deck(l0=12, m0=0, nump=256, numx=10, dt=0.01, density_np=2e22, xmax=1.0),
    ]
    out = []
    for i, d in enumerate(decks):
        st = seeded_state(d, seed=100 + i, fields=d.numy > 1)
        if d.numy == 1:
            for (l, m) in d.harmonics():
                if m > 0:
                    st.f[d.ind(l, m)] = 0
            st.fields[1:] = 0
        out.append((cfg_of(d, precision=precision), st))
    return out


def _solo(cfg, st, nsteps, collide):
    from oshun_b200 import Handle
    with Handle(**cfg) as h:
        h.upload(st.f, st.fields)
        h.step(nsteps, collisions=collide)
        return h.download()


def _batch(problems, nsteps, collide, tiles=None, autotune=False, stream=None):
    from oshun_b200 import Batch
    with Batch([c for c, _ in problems], collide=collide) as b:
        if stream is not None:
            b.set_stream(stream.cuda_stream)
        for i, (_, st) in enumerate(problems):
            b.upload(i, st.f, st.fields)
        if autotune:
            before = [b.download(i) for i in range(b.n)]
            nc, tx, ms = b.autotune(steps=1)
            assert nc in (128, 192, 256, 320) and tx in (1, 2, 4, 8) and ms > 0
            after = [b.download(i) for i in range(b.n)]
            for (f0, l0), (f1, l1) in zip(before, after):
                assert np.array_equal(f0, f1) and np.array_equal(l0, l1)
        if tiles:
            b.set_tiles(*tiles)
        b.step(nsteps)
        assert b.status() == 0
        return [b.download(i) for i in range(b.n)]


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("tiles", [None, (256, 1), (256, 2)])
def test_batch_matches_solo_runs(precision, tiles):
    problems = _mixed(precision)
    collide = [True, True, True, True, False, True]
    got = _batch(problems, 4, collide, tiles=tiles)
    for (cfg, st), col, (f, fl) in zip(problems, collide, got):
        fs, fls = _solo(cfg, st, 4, col)
        assert np.array_equal(f, fs), cfg
        assert np.array_equal(fl, fls), cfg


def test_batch_on_a_caller_stream():
    import torch
    problems = _mixed(0)
    collide = [True] * len(problems)
    stream = torch.cuda.Stream()
    got = _batch(problems, 3, collide, stream=stream)
    for (cfg, st), (f, fl) in zip(problems, got):
        fs, fls = _solo(cfg, st, 3, True)
        assert np.array_equal(f, fs) and np.array_equal(fl, fls)


def test_batch_rejects_narrow_tiles():
    from oshun_b200 import Batch, OshunError
    problems = _mixed(0)
    with Batch([c for c, _ in problems]) as b:
        with pytest.raises(OshunError):
            b.set_tiles(128, 4)       # a 256-point momentum row needs 256 threads
        assert b.tiles()[0] == 256


def test_batch_fp64_against_oracle(oracle):
    problems = _mixed(0)
    collide = [True] * len(problems)
    got = _batch(problems, 3, collide)
    for (cfg, st), (f, fl) in zip(problems, got):
        ref = oracle.steps(st, 3, 15)
        err, where = worst_rel(State(st.deck, f, fl), ref)
        assert err <= 1e-12, (cfg["l0"], cfg["m0"], err, where)


def test_batch_autotune_keeps_state():
    problems = _mixed(1)
    collide = [True] * len(problems)
    got = _batch(problems, 2, collide, autotune=True)
    for (cfg, st), (f, fl) in zip(problems, got):
        fs, fls = _solo(cfg, st, 2, True)
        assert np.array_equal(f, fs) and np.array_equal(fl, fls)


def _deck(cfg) -> Deck:
    return Deck(l0=cfg["l0"], m0=cfg["m0"], nump=cfg["nump"], numx=cfg["numx"], numy=cfg["numy"],
                NB_algorithms=cfg["NB_algorithms"], if_tridiagonal=cfg["if_tridiagonal"],
                if_implicit1D=cfg["if_implicit1D"], pmin=cfg["pmin"], pmax=cfg["pmax"], xmin=cfg["xmin"],
                xmax=cfg["xmax"], dt=cfg["dt"], small_dt=cfg["small_dt"], density_np=cfg["density_np"],
                Zeta=cfg["Zeta"])


def test_batch512_sampled(oracle):
    from oshun_b200 import Batch, workloads
    probs, meta = workloads.batch_problems()
    cfgs = [c for c, _, _, _ in probs]
    collide = [c for _, _, _, c in probs]
    with Batch(cfgs, collide=collide) as b:
        for i, (_, f, fl, _) in enumerate(probs):
            b.upload(i, f, fl)
        b.step(2)
        assert b.status() == 0
        for i in (0, 7, 131, 300, 511):
            cfg, f0, fl0, col = probs[i]
            f, fl = b.download(i)
            st = State(_deck(cfg), f0, fl0)
            fs, fls = _solo(cfg, st, 2, col)
            assert np.array_equal(f, fs) and np.array_equal(fl, fls)
            ref = oracle.steps(st, 2, 15 if col else 1)
            err, where = worst_rel(State(st.deck, f, fl), ref, floor=1e-3)
            assert err <= 1e-6, (i, err, where)
