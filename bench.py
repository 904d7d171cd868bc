"""Benchmark of the OSHUN hot path on B200: phase-space updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload weibel2d]
                    [--precision fp64|fp32] [--impl ours|reference]

One step is the reference's small-step sequence (OSHUN-1/main.cpp:77-107):
RK4 Vlasov-Maxwell stage, f00 e-e collisions, implicit f1 and f_lm
collisions.  One update is one (l,m,p,x,y) coefficient advanced one full
step.  The default workload is the 2D2V Weibel configuration (128^2 cells,
lmax = mmax = 6, np = 96): the largest single-GPU configuration, the one
whose state (616 MB per copy in FP64, 4 copies) makes %HBM meaningful.

value      device-resident throughput (state in HBM when timing starts)
e2e        the same metric through the C ABI with host buffers: every step
           uploads the state from pinned host memory, steps, downloads it
roofline   the fused RK4-stage kernel: algorithmic bytes per launch / its
           average launch time (CUDA events on the handle's stream)
cpu_baseline  the reference's own code (oracle/_ref, compiled from the OSHUN
           sources) on a bounded sample of the same workload, all host cores

N > 1 runs independent replicas, one per GPU (each workload fits one GPU and
the path needs no collective), value = sum over ranks, time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "phase-space updates/s"
UNIT = "coefficient-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="weibel2d",
                    help="weibel2d, weibel2d_64, landau1d, landau1d_large, relax1d, or batchN "
                         "(N independent uneven 1D problems in one batch, e.g. batch512)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_init():
    """One process per GPU (torchrun env); NCCL with GPUs, gloo without (the
    CPU tests of the replica logic)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def _dev():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def reduce_max(x: float, ws: int) -> float:
    """max over ranks (the timed region's length is the slowest rank's)"""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_dev())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def replica_value(units_per_rank: float, ms_total_max: float, steps: int, ws: int) -> float:
    """whole-job throughput of N independent replicas: every rank's units over
    the slowest rank's time"""
    return units_per_rank * steps * ws / (ms_total_max * 1e-3)


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# work accounting
# ----------------------------------------------------------------------------

def accounting(cfg: dict):
    """Coefficient updates per step and the algorithmic HBM bytes of one
    fused RK4-stage launch and of one full step."""
    l0, m0 = cfg["l0"], cfg["m0"]
    nh = ((m0 + 1) * (2 * l0 - m0 + 2)) // 2
    cells = cfg["numx"] * cfg["numy"]
    np_ = cfg["nump"]
    coef_updates = nh * cells * np_
    # real planes: f00 (FP64), l >= 1: 1 plane (m = 0) or 2 (m > 0)
    n_m0 = l0                       # (l,0), l >= 1
    n_cplx = nh - 1 - n_m0
    planes = n_m0 + 2 * n_cplx
    ts = 4 if cfg["precision"] == 1 else 8
    plane_elem_bytes = 8 * cells * np_ + ts * planes * cells * np_ + ts * 6 * cells
    # RK4 stages move 3, 5, 5, 3 words per element (input, Y0, Y read/write,
    # next input); the collision step reads and writes the distribution once
    stage_bytes_avg = 4 * plane_elem_bytes
    step_bytes = 16 * plane_elem_bytes + 2 * (8 * cells * np_ + ts * planes * cells * np_)
    real_dof = cells * np_ * (1 + planes)
    return dict(coef_updates=coef_updates, real_dof=real_dof, stage_bytes=stage_bytes_avg,
                step_bytes=step_bytes, planes=planes)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload: str, precision: str):
    """DRAM bytes per launch of the stage kernel from the committed ncu
    summary, scaled to this workload (null when no capture is committed)."""
    p = os.path.join(ROOT, "profiles", f"rk_stage_{workload}_{precision}.json")
    if not os.path.exists(p):
        return None
    try:
        return float(json.load(open(p))["dram_bytes_per_launch_full"])
    except (KeyError, ValueError):
        return None


# ----------------------------------------------------------------------------
# CPU baseline: the reference's own code on a bounded sample
# ----------------------------------------------------------------------------

def cpu_sample_run(workload: str, nproc: int, steps: int = 8):
    """Runs the reference build (else the C restatement) on a 16x16-cell
    sample of the workload in `nproc` parallel processes; returns
    (updates/s aggregate, kind, sample description, seconds)."""
    from oracle.cases import Deck, Oracle, REF_BIN, State, reference_available, write_case  # checker only
    from oshun_b200 import workloads

    cfg, f, fields, meta = workloads.build(workload, 0)
    sx = min(16, cfg["numx"])
    sy = min(16, cfg["numy"]) if cfg["numy"] > 1 else 1
    deck = Deck(l0=cfg["l0"], m0=max(cfg["m0"], 2) if cfg["numy"] == 1 else cfg["m0"], nump=cfg["nump"],
                numx=sx, numy=sy, NB_algorithms=cfg["NB_algorithms"], if_tridiagonal=cfg["if_tridiagonal"],
                if_implicit1D=cfg["if_implicit1D"], pmin=cfg["pmin"], pmax=cfg["pmax"], xmin=cfg["xmin"],
                xmax=cfg["xmin"] + (cfg["xmax"] - cfg["xmin"]) / (cfg["numx"] - 1) * (sx - 1),
                ymin=cfg["ymin"], ymax=cfg["ymin"] + ((cfg["ymax"] - cfg["ymin"]) / (cfg["numy"] - 1) * (sy - 1)
                                                       if cfg["numy"] > 1 else 1.0),
                dt=cfg["dt"], small_dt=cfg["small_dt"], density_np=cfg["density_np"], Zeta=cfg["Zeta"])
    st = State(deck)
    # the sample's own harmonics (m > m0 of a 1D run stay zero)
    for (l, m) in deck.harmonics():
        if m <= cfg["m0"]:
            hi = workloads.ind(l, m, cfg["m0"])
            st.f[deck.ind(l, m)] = f[hi, :sy, :sx, :]
    st.fields[:] = fields[:, :sy, :sx]
    useful = workloads.num_harmonics(cfg["l0"], cfg["m0"]) * sx * sy * cfg["nump"] * steps
    sample = f"{workload} on {sx}x{sy} cells (lmax={cfg['l0']}, mmax={cfg['m0']}, np={cfg['nump']}), {steps} step(s) per process"
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.case")
        write_case(fin, st)
        if reference_available():
            kind = "reference"
            procs = [subprocess.Popen([REF_BIN, fin, os.path.join(td, f"o{i}.case"), f"step:{steps}:15", "time"],
                                      stdout=subprocess.PIPE, text=True) for i in range(nproc)]
            times = []
            for pr in procs:
                out, _ = pr.communicate(timeout=900)
                times.append(float(out.strip().split("elapsed_s=")[-1]))
            secs = max(times)
        else:
            kind = "port"
            orc = Oracle()
            t0 = time.perf_counter()
            orc.steps(st, steps, 15)
            secs = time.perf_counter() - t0
            nproc = 1
    return useful * nproc / secs, kind, sample, secs, nproc


# ----------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------

def run_reference_arm(args, ws, rank):
    if rank != 0:
        return 0
    ncores = os.cpu_count() or 1
    vals, secs_all = [], []
    kind = sample = None
    batch = args.workload.startswith("batch")
    if batch:
        from oshun_b200 import workloads
        probs, _ = workloads.batch_problems(n=int(args.workload[len("batch"):] or 512), precision=0)
    for i in range(args.warmup + args.steps):
        if batch:
            t0 = time.perf_counter()
            r = cpu_batch_sample(probs, ncores)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "the reference build (oracle/_ref) is missing"}))
                return 0
            v, kind, sample, secs, used = r[0], r[1], r[2], time.perf_counter() - t0, min(8, ncores)
        else:
            v, kind, sample, secs, used = cpu_sample_run(args.workload, ncores, steps=1)
        if i >= args.warmup:
            vals.append(v)
            secs_all.append(secs)
    value = float(np.median(vals))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.median(secs_all)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": args.workload, "precision": "fp64",
                                        "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, ws, rank, local):
    import torch

    from oshun_b200 import Handle, workloads

    prec = 1 if args.precision == "fp32" else 0
    cfg, f, fields, meta = workloads.build(args.workload, prec)
    acct = accounting(cfg)
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    h = Handle(**cfg)
    h.set_stream(stream.cuda_stream)
    h.upload(f, fields)

    # warm-up (untimed)
    h.step(args.warmup, collisions=True)
    h.synchronize()

    # ---- device-resident timed region --------------------------------------
    sampler = ClockSampler(local)
    sampler.start()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h.step(args.steps, collisions=True)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop()
    ms_total = reduce_max(e0.elapsed_time(e1), ws)
    ms_step = ms_total / args.steps
    value = replica_value(acct["coef_updates"], ms_total, args.steps, ws)

    # ---- stage-kernel roofline: RK4-only steps (4 stage launches each) ------
    nrk = max(3, min(args.steps, 10))
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    for _ in range(nrk):
        h.rk4_step()
    r1.record(stream)
    torch.cuda.synchronize()
    launch_ms = r0.elapsed_time(r1) / (4 * nrk)
    peak, peak_kind = measured_peaks()
    achieved = acct["stage_bytes"] / (launch_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": ncu_traffic(args.workload, args.precision),
                "peak_source": peak_kind, "kernel": "rk_stage_tile_kernel (+ stage_fields_kernel)",
                "algorithmic_bytes_per_launch": acct["stage_bytes"], "avg_launch_ms": round(launch_ms, 4)}
    step_gbs = acct["step_bytes"] / (ms_step * 1e-3) / 1e9

    # ---- end to end through the C ABI with host buffers ---------------------
    hf = torch.empty(f.size * 2, dtype=torch.float64, pin_memory=True)
    hfl = torch.empty(fields.size * 2, dtype=torch.float64, pin_memory=True)
    hf.numpy().view(np.complex128)[:] = f.ravel()
    hfl.numpy().view(np.complex128)[:] = fields.ravel()
    ne = max(1, args.e2e_steps)
    h.upload_ptr(hf.data_ptr(), hfl.data_ptr())
    h.step(1, collisions=True)
    h.download_ptr(hf.data_ptr(), hfl.data_ptr())
    torch.cuda.synchronize()
    barrier(ws)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for _ in range(ne):
        h.upload_ptr(hf.data_ptr(), hfl.data_ptr())
        h.step(1, collisions=True)
        h.download_ptr(hf.data_ptr(), hfl.data_ptr())
    q1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_max(q0.elapsed_time(q1), ws) / ne
    e2e_value = acct["coef_updates"] * ws / (e2e_ms * 1e-3)
    state_bytes = int(f.nbytes + fields.nbytes)
    h.close()

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, kind, sample, secs, used = cpu_sample_run(args.workload, os.cpu_count() or 1)
        cpu = {"value": v, "unit": UNIT, "cores": used, "kind": kind, "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == 0 else "f32+f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "precision": args.precision,
                       "cells": cfg["numx"] * cfg["numy"], "lmax": cfg["l0"], "mmax": cfg["m0"],
                       "np": cfg["nump"], "coefficients": acct["coef_updates"], "real_dof": acct["real_dof"],
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (4 state copies of "
                             f"{acct['stage_bytes'] / 4 / 1e6:.0f} MB each; L2 is 126 MB)",
                       "step_hbm_GBps": round(step_gbs, 1)},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "ms_per_step": e2e_ms},
            "roofline": roofline,
            # per step: 4 RK4 stages (the stage kernel and its field kernel each),
            # the clock advance, the collision kernel, the clock commit
            "gpu_launches": 11 * args.steps,
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    return 0


def batch_accounting(probs):
    coefs = 0
    step_bytes = 0
    for cfg, _, _, col in probs:
        a = accounting(cfg)
        coefs += a["coef_updates"]
        # RK4 16 words per element; the collision step 2 more when it runs
        step_bytes += a["step_bytes"] if col else 4 * a["stage_bytes"]
    return coefs, step_bytes


def cpu_batch_sample(probs, nproc: int):
    """The reference's own code on 8 sampled problems of the batch (those with
    lmax >= 3, the reference's smallest supported case; 1D runs carry m <= 2
    in the reference, only the batch's own harmonics are counted), one step
    each, in parallel processes; returns (updates/s, kind, sample)."""
    from oracle.cases import Deck, REF_BIN, State, reference_available, write_case  # checker only
    from oshun_b200 import workloads
    if not reference_available():
        return None
    pick = [i for i, (c, _, _, _) in enumerate(probs) if c["l0"] >= 3][:max(1, min(8, nproc))]
    useful = 0
    with tempfile.TemporaryDirectory() as td:
        procs = []
        for i in pick:
            cfg, f, fields, col = probs[i]
            d = Deck(l0=cfg["l0"], m0=2, nump=cfg["nump"], numx=cfg["numx"], numy=1, pmin=cfg["pmin"],
                     pmax=cfg["pmax"], xmin=cfg["xmin"], xmax=cfg["xmax"], dt=cfg["dt"], small_dt=cfg["small_dt"],
                     density_np=cfg["density_np"])
            st = State(d)
            for l in range(cfg["l0"] + 1):
                st.f[d.ind(l, 0)] = f[l]
            st.fields[:] = fields
            fin = os.path.join(td, f"in{i}.case")
            write_case(fin, st)
            procs.append(subprocess.Popen([REF_BIN, fin, os.path.join(td, f"o{i}.case"),
                                           f"step:1:{15 if col else 1}", "time"], stdout=subprocess.PIPE, text=True))
            useful += workloads.num_harmonics(cfg["l0"], 0) * cfg["numx"] * cfg["nump"]
        secs = max(float(p.communicate(timeout=900)[0].strip().split("elapsed_s=")[-1]) for p in procs)
    return useful / secs, "reference", f"{len(pick)} problems of the batch with lmax >= 3, 1 step each, one process each"


def run_batch(args, ws, rank, local):
    """Batch of N independent uneven 1D problems (workloads.batch_problems),
    FP32 bulk by default: one captured graph per step, tiles autotuned on the
    batch itself before timing."""
    import torch
    from oshun_b200 import Batch, workloads
    torch.cuda.set_device(local)
    n = int(args.workload[len("batch"):] or 512)
    prec = 0 if args.precision == "fp64" else 1
    probs, meta = workloads.batch_problems(n=n, precision=prec, seed=2024 + rank)
    coefs, step_bytes = batch_accounting(probs)
    b = Batch([c for c, _, _, _ in probs], collide=[c for _, _, _, c in probs])
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    for i, (_, f, fl, _) in enumerate(probs):
        b.upload(i, f, fl)
    nc, tx, tune_ms = b.autotune(steps=2)
    b.step(args.warmup)
    torch.cuda.synchronize()
    barrier(ws)
    sampler = ClockSampler(local)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms_total = reduce_max(e0.elapsed_time(e1), ws)
    ms_step = ms_total / args.steps
    value = replica_value(coefs, ms_total, args.steps, ws)
    assert b.status() == 0
    peak, peak_kind = measured_peaks()
    achieved = step_bytes / (ms_step * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                "kernel": "whole step (batched stage and collision kernels)",
                "algorithmic_bytes_per_step": step_bytes}
    # end to end: every step uploads every problem's state, steps, downloads it
    ne = max(1, args.e2e_steps)
    state_bytes = sum(int(f.nbytes + fl.nbytes) for _, f, fl, _ in probs)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for _ in range(ne):
        for i, (_, f, fl, _) in enumerate(probs):
            b.upload(i, f, fl)
        b.step(1)
        for i in range(n):
            b.download(i)
    q1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_max(q0.elapsed_time(q1), ws) / ne
    b.close()
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        r = cpu_batch_sample(probs, os.cpu_count() or 1)
        if r:
            cpu = {"value": r[0], "unit": UNIT, "cores": min(8, os.cpu_count() or 1), "kind": r[1], "sample": r[2]}
    if rank == 0:
        # per step: 4 batched stages (stage kernel + field kernel each), 2 clock
        # kernels, one collision launch per group of equal ceil(nump/32) and
        # the same side of 8 resident collision CTAs per SM (the library's grouping)
        def ctas_per_sm(c):
            np_, l0 = c["nump"], c["l0"]
            smem = 8 * (4 + 4 * np_ + max(9 * np_, 2 * l0 * np_))
            return min(16, max(1, (228 * 1024) // (smem + 1024)))
        nsteps_groups = 8 + 2 + len({((c["nump"] + 31) // 32, ctas_per_sm(c) >= 8) for c, _, _, col in probs if col})
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == 0 else "f32+f64", "data": "synthetic",
            "config": {"workload": args.workload, "precision": args.precision, "problems": n,
                       "coefficients": coefs, "seed": meta["seed"], "stage_threads": nc, "tile_cells": tx,
                       "autotune_ms_per_step": round(tune_ms, 4),
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                       "l2": "inputs larger than L2"},
            "e2e": {"value": coefs * ws / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "ms_per_step": e2e_ms},
            "roofline": roofline,
            "gpu_launches": nsteps_groups * args.steps,
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            return run_reference_arm(args, ws, rank)
        if args.workload.startswith("batch"):
            return run_batch(args, ws, rank, local)
        return run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
