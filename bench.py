#!/usr/bin/env python
"""Benchmark of the B200 hot path: cell-steps/s of the tracer step, mixed FP32/FP64 vs plain FP64.

One step = one tracer advection-diffusion step, i.e. do_advection_3d (HALFSPLIT, SUPERBEE in
u, v and w) followed by the implicit vertical-diffusion solve (the body of do_salinity,
salinity.F90:301-389), on the rotation recipe (closed flat basin, solid-body rotation, Gaussian
blob + seeded noise) at 2048 x 2048 x 50. A cell-step is one interior cell advanced by one step.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line (rank 0). The default arm runs the CUDA library; `--impl reference` times
the CPU restatement of the reference routines (the oracle, OpenMP over all host cores) on a
bounded sample of the same workload. Multi-GPU runs (torchrun) are weak-scaled replicas: every
rank advances its own 2048 x 2048 x 50 basin; the tracer step of a closed basin has no exchange.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s mixed-prec vs plain FP64 on 1 B200 at stated err; adjoint/fwd ratio"
UNIT = "cell-steps/s"
# algorithmic words per interior cell per launch of each stage (read + write, each field once)
STAGE_WORDS = {"adv_split_u": 6, "adv_split_v": 6, "adv_split_w": 5, "tracer_vdiff": 4, "adv_finalise": 4,
               "tracer_fused_uv": 8, "tracer_fused_wvu": 9}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--kmax", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            pk = json.load(fh)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
        return False

    def summary(self):
        rows = []
        for line in (getattr(self, "out", "") or "").strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    """CPU restatement (oracle) on a bounded sample of the workload, all host threads."""
    if rank != 0:
        return
    import numpy as np

    import oracle
    from code_b200 import cases

    snx, sny = min(args.nx, 1024), min(args.ny, 1024)
    c = cases.tracer_rotation(nx=snx, ny=sny, kmax=args.kmax, depth=50.0, dx=1000.0, dt=60.0, sigma_cells=32.0)
    p = c.par
    o = oracle.Oracle(c.grid)
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    f = c["f"].copy()
    arr = [c[n] for n in names]
    run = lambda n: o.tracer_steps(c.masks(), n, p["dt"], f, *arr, 2, 4, 4, 0.0, 1.0, 0.0)  # noqa: E731
    run(max(args.warmup, 0))
    t0 = time.perf_counter()
    run(args.steps)
    el = time.perf_counter() - t0
    cells = snx * sny * args.kmax
    v = cells * args.steps / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "tracer step (do_advection_3d HALFSPLIT SUPERBEE + implicit vertical diffusion), "
                               "rotation recipe, closed flat basin", "nx": args.nx, "ny": args.ny,
                   "kmax": args.kmax, "sample": f"{snx}x{sny}x{args.kmax} per step"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{snx}x{sny}x{args.kmax}, {args.steps} steps after {args.warmup} warm-up"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def cpu_baseline_sample(args):
    import oracle
    from code_b200 import cases

    snx, sny = min(args.nx, 1024), min(args.ny, 512)
    c = cases.tracer_rotation(nx=snx, ny=sny, kmax=args.kmax, depth=50.0, dx=1000.0, dt=60.0, sigma_cells=32.0)
    p = c.par
    o = oracle.Oracle(c.grid)
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    f = c["f"].copy()
    arr = [c[n] for n in names]
    o.tracer_steps(c.masks(), 1, p["dt"], f, *arr, 2, 4, 4, 0.0, 1.0, 0.0)
    n, t0 = 0, time.perf_counter()
    while True:
        o.tracer_steps(c.masks(), 1, p["dt"], f, *arr, 2, 4, 4, 0.0, 1.0, 0.0)
        n += 1
        el = time.perf_counter() - t0
        if el > 10.0 or n >= 50:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": snx * sny * args.kmax * n / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle FP64 tracer step on {snx}x{sny}x{args.kmax}, {n} steps ({el:.1f} s)"}


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    import torch
    import torch.distributed as dist

    from code_b200 import cases
    from code_b200.getm import Context

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    res = {}
    variants = {}
    for key, dt_ in (("fp64", torch.float64), ("mixed", torch.float32)):
        g, fld, par = cases.tracer_rotation_device(args.nx, args.ny, args.kmax, dtype=dt_, seed=1 + rank)
        ctx = Context(g, stream)
        ctx.init_advection(fld["az"], fld["au"], fld["av"], fld["ax"])
        variants[key] = (g, fld, par, ctx)
    steps_done = {}

    def step(key):
        g, fld, par, ctx = variants[key]
        cast = float
        ctx.tracer_step(cast(par["dt"]), fld["f"], *[fld[n] for n in names], 2, 4, 4, 0.0, 1.0, 0.0)
        steps_done[key] = steps_done.get(key, 0) + 1

    cells = args.nx * args.ny * args.kmax
    clocks = None
    for key in ("fp64", "mixed"):
        for _ in range(args.warmup):
            step(key)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as cs:
            e0.record(stream)
            for _ in range(args.steps):
                step(key)
            e1.record(stream)
            barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        res[key] = {"ms": ms, "value": world * cells * args.steps / (ms / 1e3)}
        if key == "mixed":
            clocks = cs.summary()
    # stated error of the mixed variant against FP64 after the same number of steps
    f64 = variants["fp64"][1]["f"]
    f32 = variants["mixed"][1]["f"]
    err = None
    if steps_done["fp64"] == steps_done["mixed"]:
        d = (f32.double() - f64).abs()
        err = {"field": "tracer", "max_abs": float(d.max()), "rms": float(d.pow(2).mean().sqrt()),
               "amplitude": float(f64.abs().max()), "steps": steps_done["fp64"]}
    # per-stage timers over K more steps of the mixed variant (dominant kernel roofline)
    ctx = variants["mixed"][3]
    ctx.timers(enable=True, reset=True)
    for _ in range(args.steps):
        step("mixed")
    torch.cuda.synchronize()
    tim = ctx.timers(enable=False, reset=True)
    launches = sum(n for _, n in tim.values())
    top = max(tim.items(), key=lambda kv: kv[1][0])
    top_name, (top_ms, top_n) = top
    wb = 4
    alg_bytes = STAGE_WORDS.get(top_name, 0) * cells * wb
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (top_ms / top_n / 1e3) / 1e9
    # end-to-end through the C ABI with host buffers: per step H2D of the tracer, step, D2H
    g, fld, par, ctx = variants["mixed"]
    hbuf = torch.empty_like(fld["f"], device="cpu").pin_memory()
    hbuf.copy_(fld["f"])
    barrier()
    k2 = max(3, args.steps // 4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k2):
        fld["f"].copy_(hbuf, non_blocking=True)
        step("mixed")
        hbuf.copy_(fld["f"], non_blocking=True)
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    nbytes = fld["f"].numel() * fld["f"].element_size()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_sample(args)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}
    if rank == 0:
        out = {
            "metric": METRIC, "value": res["mixed"]["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["mixed"]["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "tracer step (do_advection_3d HALFSPLIT SUPERBEE + implicit vertical diffusion), "
                                   "rotation recipe, closed flat basin", "nx": args.nx, "ny": args.ny,
                       "kmax": args.kmax, "l2": "inputs larger than L2 (FP32 field 0.84 GB, FP64 1.7 GB)",
                       "parallelism": f"replicas x{world}"},
            "plain_fp64": {"value": res["fp64"]["value"], "ms_per_step": res["fp64"]["ms"] / args.steps},
            "mixed_over_fp64": res["mixed"]["value"] / res["fp64"]["value"],
            "err_vs_fp64": err,
            "adjoint_fwd_ratio": None,
            "gpu_launches": launches,
            "stage_ms_per_step": {k: v[0] / args.steps for k, v in tim.items()},
            "roofline": {"bound": "hbm", "kernel": top_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                         "alg_bytes_per_launch": alg_bytes},
            "e2e": {"value": world * cells * k2 / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes},
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out), flush=True)
    for key in variants:
        variants[key][3].close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
