"""Benchmark of the OSHUN hot path on B200: phase-space updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload weibel2d]
                    [--precision fp64|fp32] [--impl ours|reference] [--no-forms]

One step is the reference's small-step sequence (OSHUN-1/main.cpp:77-107):
RK4 Vlasov-Maxwell stage, f00 e-e collisions, implicit f1 and f_lm
collisions (the Landau workloads are collisionless: RK4 only).  One update
is one (l,m,p,x,y) coefficient advanced one full step.  The default workload
is the 2D2V Weibel configuration (128^2 cells, lmax = mmax = 6, np = 96):
the largest single-GPU configuration, the one whose state (616 MB per copy
in FP64, 4 copies) makes %HBM meaningful.

value      device-resident throughput (state in HBM when timing starts)
e2e        the same metric through the C ABI with host buffers: every step
           uploads the state from pinned host memory, steps, downloads it
roofline   the fused RK4-stage kernel: algorithmic bytes per launch / its
           average launch time (CUDA events on the handle's stream)
forms      (1 GPU, default workload) the other forms of the metric on the
           same box: the FP32/FP64 split Weibel run, the 512-problem FP32
           batch and the large FP64 1D Landau run, each with its value,
           ms/step, roofline fraction and error against the FP64 GPU path,
           and the time of one adjoint gradient of the sensitivity case
cpu_baseline  the reference's own code (oracle/_ref, compiled from the OSHUN
           sources) on a bounded sample of the same workload, all host cores;
           per useful coefficient and raw (the reference's guard cells and
           extra harmonics included)

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
    ap.add_argument("--no-forms", action="store_true")
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
    """nvidia-smi sampled every 20 ms from before the warm-up; stop() keeps
    the samples inside the timed window (host wall clock around the timed
    region; the nearest sample when the window is shorter than the period)."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.window = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # wait (bounded) for the first sample, so the timed region is covered
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
            time.sleep(0.02)

    def mark(self, t0: float, t1: float):
        self.window = (t0, t1)

    @staticmethod
    def _epoch(ts: str):
        import datetime
        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(ts.strip(), fmt).timestamp()
            except ValueError:
                pass
        return None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                rows.append((self._epoch(parts[0]), float(parts[2]), float(parts[3]),
                             {nm for nm, v in zip(names, parts[6:10]) if v.lower() in ("active", "1")}))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sel = rows
        if self.window is not None and all(r[0] is not None for r in rows):
            t0, t1 = self.window
            sel = [r for r in rows if t0 <= r[0] <= t1]
            if not sel:   # window shorter than the sampling period: the nearest sample
                mid = 0.5 * (t0 + t1)
                sel = [min(rows, key=lambda r: abs(r[0] - mid))]
        reasons = set()
        for r in sel:
            reasons |= r[3]
        return {"sm_mhz": float(np.median([r[1] for r in sel])), "sm_max_mhz": max(r[2] for r in sel),
                "reasons": sorted(reasons), "samples": len(sel), "samples_total": len(rows)}


# ----------------------------------------------------------------------------
# work accounting
# ----------------------------------------------------------------------------

def collisional(workload: str) -> bool:
    """The Landau configurations are collisionless (RK4 only); every other
    workload runs the full small step."""
    return not workload.startswith("landau")


def accounting(cfg: dict, collisions: bool = True):
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
    step_bytes = 16 * plane_elem_bytes
    collide_bytes = 2 * (8 * cells * np_ + ts * planes * cells * np_)
    if collisions:
        step_bytes += collide_bytes
    real_dof = cells * np_ * (1 + planes)
    return dict(coef_updates=coef_updates, real_dof=real_dof, stage_bytes=stage_bytes_avg,
                step_bytes=step_bytes, collide_bytes=collide_bytes, planes=planes)


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

NBC = 4   # the reference's guard cells per side (RKLevel, OSHUN-1/def-Input.cpp:156-164)


def cpu_sample_run(workload: str, nproc: int, steps: int = 8):
    """Runs the reference build (else the C restatement) on a 16x16-cell
    sample of the workload in `nproc` parallel processes; returns
    (updates/s per useful coefficient, kind, sample description, seconds,
    processes, raw updates/s).  Raw counts every coefficient the reference
    advances: its 4 guard cells per side and, for 1D runs, the m <= 2
    harmonics and 4 y rows it needs."""
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
    ny_ref = sy if sy > 1 else NBC
    raw = deck.nh * (sx + 2 * NBC) * (ny_ref + 2 * NBC) * cfg["nump"] * steps
    mask = 15 if collisional(workload) else 1
    sample = (f"{workload} on {sx}x{sy} cells (lmax={cfg['l0']}, mmax={cfg['m0']}, np={cfg['nump']}), "
              f"{steps} step(s) per process")
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.case")
        write_case(fin, st)
        if reference_available():
            kind = "reference"
            procs = [subprocess.Popen([REF_BIN, fin, os.path.join(td, f"o{i}.case"), f"step:{steps}:{mask}", "time"],
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
            orc.steps(st, steps, mask)
            secs = time.perf_counter() - t0
            nproc = 1
            raw = useful
    return useful * nproc / secs, kind, sample, secs, nproc, raw * nproc / secs


# ----------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------

def run_reference_arm(args, ws, rank):
    if rank != 0:
        return 0
    ncores = os.cpu_count() or 1
    vals, raws, secs_all = [], [], []
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
            v, kind, sample, secs, used, raw = r[0], r[1], r[2], time.perf_counter() - t0, min(8, ncores), r[3]
        else:
            v, kind, sample, secs, used, raw = cpu_sample_run(args.workload, ncores, steps=1)
        if i >= args.warmup:
            vals.append(v)
            raws.append(raw)
            secs_all.append(secs)
    value = float(np.median(vals))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.median(secs_all)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": args.workload, "precision": "fp64",
                                        "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": kind, "sample": sample,
                         "raw_value": float(np.median(raws)),
                         "raw_note": "every coefficient the reference advances (guard cells, extra harmonics)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def time_handle(h, stream, steps: int, warmup: int, collisions: bool, ws: int, sampler=None):
    """Device-resident timing of `steps` small steps after `warmup` untimed
    ones: CUDA events on the handle's stream, barrier + synchronize on both
    sides, max over ranks.  Returns the total ms."""
    import torch
    h.step(warmup, collisions=collisions)
    h.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall = time.time()
    e0.record(stream)
    h.step(steps, collisions=collisions)
    e1.record(stream)
    torch.cuda.synchronize()
    if sampler is not None:
        sampler.mark(t_wall, time.time())
    barrier(ws)
    return reduce_max(e0.elapsed_time(e1), ws)


def stage_roofline(h, stream, acct: dict, nrk: int, kernel: str, traffic=None) -> dict:
    """Average stage launch (stage kernel + its field kernel) over RK4-only
    steps (4 launches each), against the measured HBM peak."""
    import torch
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    for _ in range(nrk):
        h.rk4_step()
    r1.record(stream)
    torch.cuda.synchronize()
    launch_ms = r0.elapsed_time(r1) / (4 * nrk)
    peak, peak_kind = measured_peaks()
    achieved = acct["stage_bytes"] / (launch_ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind, "kernel": kernel,
            "algorithmic_bytes_per_launch": acct["stage_bytes"], "avg_launch_ms": round(launch_ms, 4)}


def rel_errors(a_f, a_fl, b_f, b_fl, floor: float = 1e-6):
    """Error of the state a against the state b: the max over harmonics and
    fields of the relative L2 error, each norm floored at `floor` times the
    largest harmonic (or field) norm, so that a harmonic that is zero up to
    rounding in b is measured against the state's own scale; and the relative
    L2 error of the whole distribution.  Returns (worst, where, state)."""
    worst, where = 0.0, None
    topf = max(float(np.linalg.norm(b_f[i])) for i in range(b_f.shape[0]))
    topl = max(float(np.linalg.norm(b_fl[i])) for i in range(6))
    for i in range(b_f.shape[0]):
        nb = max(float(np.linalg.norm(b_f[i])), floor * topf)
        if nb > 0:
            e = float(np.linalg.norm(a_f[i] - b_f[i])) / nb
            if e > worst:
                worst, where = e, f"harmonic {i}"
    for i in range(6):
        nb = max(float(np.linalg.norm(b_fl[i])), floor * topl)
        if nb > 0:
            e = float(np.linalg.norm(a_fl[i] - b_fl[i])) / nb
            if e > worst:
                worst, where = e, f"field {i}"
    nf = float(np.linalg.norm(b_f))
    state = float(np.linalg.norm(a_f - b_f)) / nf if nf > 0 else 0.0
    return worst, where, state


def form_single(workload: str, prec: int, steps: int, warmup: int, stream, err_steps: int = 2) -> dict:
    """One more single-problem form on this GPU: value, ms/step, stage
    roofline and (FP32 split) the error against the FP64 GPU path after
    err_steps steps from the same initial state."""
    from oshun_b200 import Handle, workloads
    col = collisional(workload)
    cfg, f, fields, _ = workloads.build(workload, prec)
    acct = accounting(cfg, col)
    with Handle(**cfg) as h:
        h.set_stream(stream.cuda_stream)
        h.upload(f, fields)
        ms_total = time_handle(h, stream, steps, warmup, col, 1)
        roof = stage_roofline(h, stream, acct, max(3, min(steps, 10)), "rk_stage_tile_kernel (+ stage_fields_kernel)")
    ms_step = ms_total / steps
    peak, _ = measured_peaks()
    out = {"workload": workload, "precision": "fp32" if prec else "fp64", "collisions": col,
           "value": acct["coef_updates"] * steps / (ms_total * 1e-3), "unit": UNIT, "ms_per_step": ms_step,
           "roofline": {"frac": roof["frac"], "achieved": roof["achieved"], "peak": peak, "unit": "GB/s",
                        "kernel": "stage", "avg_launch_ms": roof["avg_launch_ms"]},
           "step_hbm_frac": round(acct["step_bytes"] / (ms_step * 1e-3) / 1e9 / peak, 4),
           "coefficients": acct["coef_updates"]}
    if prec == 1:
        cfg64 = dict(cfg, precision=0)
        with Handle(**cfg64) as a, Handle(**cfg) as b:
            for h in (a, b):
                h.set_stream(stream.cuda_stream)
                h.upload(f, fields)
                h.step(err_steps, collisions=col)
            fa, fla = a.download()
            fb, flb = b.download()
        e, where, st = rel_errors(fb, flb, fa, fla)
        out["max_rel_err_vs_fp64"] = e
        out["max_rel_err_at"] = where
        out["state_rel_err_vs_fp64"] = st
        out["err_norm_floor"] = "1e-6 of the largest harmonic / field norm"
        out["err_steps"] = err_steps
    return out


def form_adjoint(stream, nsteps: int = 500, every: int = 50, cell: int = 256) -> dict:
    """The sensitivity configuration (1D, nx = 512, lmax = 2, np = 128): one
    gradient of the time-integrated heat flux of one cell with respect to
    every cell's initial temperature, forward and checkpointed backward
    through the adjoint kernels, timed with CUDA events; FP64 and the FP32
    bulk form (its gradient's largest deviation from the FP64 one, relative
    to the largest FP64 component)."""
    import torch
    from oshun_b200 import workloads
    from oshun_b200.adjoint import Run, StepsWithCheckpoints, heat_flux_weight
    cfg, tau, _ = workloads.sensitivity1d()
    w = heat_flux_weight(cfg, cell)

    def timed(prec):
        run = Run(**dict(cfg, precision=prec))

        def grad_once():
            t = torch.tensor(tau, device="cuda").requires_grad_(True)
            y0 = workloads.sensitivity_state(cfg, t)
            Q = StepsWithCheckpoints.apply(y0, run, nsteps, every, w)
            Q.backward()
            return t.grad

        with torch.cuda.stream(stream):
            grad_once()                      # warm-up
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g = grad_once()
            e1.record(stream)
            torch.cuda.synchronize()
        run.close()
        return e0.elapsed_time(e1), g.detach().cpu().numpy()

    ms, g = timed(0)
    ms32, g32 = timed(1)
    coefs = (cfg["l0"] + 1) * cfg["numx"] * cfg["nump"]
    scale = float(np.max(np.abs(g)))
    return {"workload": "sensitivity1d (nx=512, lmax=2, np=128)", "precision": "fp64", "steps": nsteps,
            "checkpoint_every": every, "ms_per_gradient": ms,
            "forward_steps_per_gradient": 2 * nsteps - nsteps // every, "vjp_steps_per_gradient": nsteps,
            "value": coefs * nsteps / (ms * 1e-3), "unit": UNIT + " (forward steps of the gradient's trajectory)",
            "grad_finite": bool(np.isfinite(g).all()),
            "fp32_bulk": {"ms_per_gradient": ms32, "value": coefs * nsteps / (ms32 * 1e-3),
                          "max_dev_vs_fp64_grad": float(np.max(np.abs(g32 - g))) / scale if scale > 0 else None}}


def run_ours(args, ws, rank, local):
    import torch

    from oshun_b200 import Handle, workloads

    prec = 1 if args.precision == "fp32" else 0
    col = collisional(args.workload)
    cfg, f, fields, meta = workloads.build(args.workload, prec)
    acct = accounting(cfg, col)
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    h = Handle(**cfg)
    h.set_stream(stream.cuda_stream)
    h.upload(f, fields)

    # clocks sampled from before the warm-up; the timed window is marked
    sampler = ClockSampler(local)
    sampler.start()
    # ---- device-resident timed region --------------------------------------
    ms_total = time_handle(h, stream, args.steps, args.warmup, col, ws, sampler)
    ms_step = ms_total / args.steps
    value = replica_value(acct["coef_updates"], ms_total, args.steps, ws)

    # ---- stage-kernel roofline: RK4-only steps (4 stage launches each) ------
    roofline = stage_roofline(h, stream, acct, max(3, min(args.steps, 10)),
                              "rk_stage_tile_kernel (+ stage_fields_kernel)",
                              ncu_traffic(args.workload, args.precision))
    peak = roofline["peak"]
    step_gbs = acct["step_bytes"] / (ms_step * 1e-3) / 1e9

    # ---- end to end through the C ABI with host buffers ---------------------
    hf = torch.empty(f.size * 2, dtype=torch.float64, pin_memory=True)
    hfl = torch.empty(fields.size * 2, dtype=torch.float64, pin_memory=True)
    hf.numpy().view(np.complex128)[:] = f.ravel()
    hfl.numpy().view(np.complex128)[:] = fields.ravel()
    ne = max(1, args.e2e_steps)
    h.upload_ptr(hf.data_ptr(), hfl.data_ptr())
    h.step(1, collisions=col)
    h.download_ptr(hf.data_ptr(), hfl.data_ptr())
    torch.cuda.synchronize()
    barrier(ws)
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for _ in range(ne):
        h.upload_ptr(hf.data_ptr(), hfl.data_ptr())
        h.step(1, collisions=col)
        h.download_ptr(hf.data_ptr(), hfl.data_ptr())
    q1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_max(q0.elapsed_time(q1), ws) / ne
    e2e_value = acct["coef_updates"] * ws / (e2e_ms * 1e-3)
    state_bytes = int(f.nbytes + fields.nbytes)
    h.close()
    clocks = sampler.stop()

    # ---- the other forms of the metric on this GPU (1 GPU, default workload) --
    forms = None
    if ws == 1 and not args.no_forms and args.workload == "weibel2d" and prec == 0:
        forms = {}
        fw = min(args.warmup, 3)
        forms["fp32_split"] = form_single("weibel2d", 1, args.steps, fw, stream)
        forms["fp32_split"]["speedup_vs_fp64"] = forms["fp32_split"]["value"] / value
        forms["landau1d_large"] = form_single("landau1d_large", 0, args.steps, fw, stream)
        forms["batch512"] = measure_batch(512, 1, args.steps, fw, stream, local, error_check=True)
        forms["batch512"].pop("_probs")
        forms["adjoint_sensitivity"] = form_adjoint(stream)
        forms["batch512"]["speedup_vs_fp64"] = forms["batch512"]["value"] / value

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, kind, sample, secs, used, raw = cpu_sample_run(args.workload, os.cpu_count() or 1)
        cpu = {"value": v, "unit": UNIT, "cores": used, "kind": kind, "sample": sample, "raw_value": raw,
               "raw_note": "every coefficient the reference advances (guard cells, extra harmonics)"}

    if rank == 0:
        # per step: 4 RK4 stages (the stage kernel and its field kernel each),
        # the clock advance and, with collisions, the collision kernel and the clock commit
        launches_per_step = 9 + (2 if col else 0)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == 0 else "f32+f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "precision": args.precision, "collisions": col,
                       "cells": cfg["numx"] * cfg["numy"], "lmax": cfg["l0"], "mmax": cfg["m0"],
                       "np": cfg["nump"], "coefficients": acct["coef_updates"], "real_dof": acct["real_dof"],
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (4 state copies of "
                             f"{acct['stage_bytes'] / 4 / 1e6:.0f} MB each; L2 is 126 MB)",
                       "step_hbm_GBps": round(step_gbs, 1), "step_hbm_frac": round(step_gbs / peak, 4)},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "ms_per_step": e2e_ms},
            "roofline": roofline,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if forms is not None:
            line["forms"] = forms
        print(json.dumps(line), flush=True)
    return 0


def batch_accounting(probs):
    coefs = 0
    step_bytes = 0
    for cfg, _, _, col in probs:
        a = accounting(cfg, bool(col))
        coefs += a["coef_updates"]
        step_bytes += a["step_bytes"]
    return coefs, step_bytes


def cpu_batch_sample(probs, nproc: int):
    """The reference's own code on 8 sampled problems of the batch (those with
    lmax >= 3, the reference's smallest supported case; 1D runs carry m <= 2
    in the reference, only the batch's own harmonics are counted), one step
    each, in parallel processes; returns (updates/s, kind, sample, raw
    updates/s)."""
    from oracle.cases import Deck, REF_BIN, State, reference_available, write_case  # checker only
    from oshun_b200 import workloads
    if not reference_available():
        return None
    pick = [i for i, (c, _, _, _) in enumerate(probs) if c["l0"] >= 3][:max(1, min(8, nproc))]
    useful = raw = 0
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
            raw += d.nh * (cfg["numx"] + 2 * NBC) * (NBC + 2 * NBC) * cfg["nump"]
        secs = max(float(p.communicate(timeout=900)[0].strip().split("elapsed_s=")[-1]) for p in procs)
    return (useful / secs, "reference", f"{len(pick)} problems of the batch with lmax >= 3, 1 step each, one process each",
            raw / secs)


def measure_batch(n: int, prec: int, steps: int, warmup: int, stream, local: int, ws: int = 1, rank: int = 0,
                  error_check: bool = False, sampler=None, e2e_steps: int = 0) -> dict:
    """Batch of n independent uneven 1D problems (workloads.batch_problems):
    one captured graph per step, tiles autotuned on the batch itself before
    timing.  With error_check, 8 sampled problems of the batch after 2 steps
    from their initial states against FP64 single-problem runs."""
    import torch
    from oshun_b200 import Batch, Handle, workloads
    probs, meta = workloads.batch_problems(n=n, precision=prec, seed=2024 + rank)
    coefs, step_bytes = batch_accounting(probs)
    b = Batch([c for c, _, _, _ in probs], collide=[c for _, _, _, c in probs])
    b.set_stream(stream.cuda_stream)
    for i, (_, f, fl, _) in enumerate(probs):
        b.upload(i, f, fl)
    nc, tx, tune_ms = b.autotune(steps=2)
    b.step(warmup)
    torch.cuda.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall = time.time()
    e0.record(stream)
    b.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if sampler is not None:
        sampler.mark(t_wall, time.time())
    ms_total = reduce_max(e0.elapsed_time(e1), ws)
    ms_step = ms_total / steps
    assert b.status() == 0
    peak, peak_kind = measured_peaks()
    achieved = step_bytes / (ms_step * 1e-3) / 1e9
    out = {"workload": f"batch{n}", "precision": "fp32" if prec else "fp64", "problems": n,
           "value": replica_value(coefs, ms_total, steps, ws), "unit": UNIT, "ms_per_step": ms_step,
           "coefficients": coefs, "seed": meta["seed"], "stage_threads": nc, "tile_cells": tx,
           "autotune_ms_per_step": round(tune_ms, 4),
           "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                        "kernel": "whole step (batched stage and collision kernels)",
                        "algorithmic_bytes_per_step": step_bytes}}
    if e2e_steps > 0:
        ne = e2e_steps
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
        out["e2e"] = {"value": coefs * ws / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                      "d2h_bytes_per_step": state_bytes, "ms_per_step": e2e_ms}
    if error_check and prec == 1:
        pick = list(range(0, n, max(1, n // 8)))[:8]
        for i, (_, f, fl, _) in enumerate(probs):
            b.upload(i, f, fl)
        b.step(2)
        worst, where, wstate = 0.0, None, 0.0
        for i in pick:
            cfg, f, fl, col = probs[i]
            fb, flb = b.download(i)
            with Handle(**dict(cfg, precision=0)) as h:
                h.set_stream(stream.cuda_stream)
                h.upload(f, fl)
                h.step(2, collisions=bool(col))
                fa, fla = h.download()
            e, w, st = rel_errors(fb, flb, fa, fla)
            wstate = max(wstate, st)
            if e > worst:
                worst, where = e, f"problem {i}, {w}"
        out["max_rel_err_vs_fp64"] = worst
        out["max_rel_err_at"] = where
        out["state_rel_err_vs_fp64"] = wstate
        out["err_norm_floor"] = "1e-6 of the largest harmonic / field norm"
        out["err_steps"] = 2
        out["err_sample"] = f"problems {pick}"
    b.close()
    out["_probs"] = probs
    return out


def run_batch(args, ws, rank, local):
    """Batch of N independent uneven 1D problems, FP32 bulk by default."""
    import torch
    torch.cuda.set_device(local)
    n = int(args.workload[len("batch"):] or 512)
    prec = 0 if args.precision == "fp64" else 1
    stream = torch.cuda.Stream()
    sampler = ClockSampler(local)
    sampler.start()
    r = measure_batch(n, prec, args.steps, args.warmup, stream, local, ws, rank, sampler=sampler,
                      e2e_steps=max(1, args.e2e_steps))
    clocks = sampler.stop()
    probs = r.pop("_probs")
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        c = cpu_batch_sample(probs, os.cpu_count() or 1)
        if c:
            cpu = {"value": c[0], "unit": UNIT, "cores": min(8, os.cpu_count() or 1), "kind": c[1], "sample": c[2],
                   "raw_value": c[3]}
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
            "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == 0 else "f32+f64", "data": "synthetic",
            "config": {"workload": args.workload, "precision": args.precision, "problems": n,
                       "coefficients": r["coefficients"], "seed": r["seed"], "stage_threads": r["stage_threads"],
                       "tile_cells": r["tile_cells"], "autotune_ms_per_step": r["autotune_ms_per_step"],
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                       "l2": "inputs larger than L2"},
            "e2e": r["e2e"],
            "roofline": r["roofline"],
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
