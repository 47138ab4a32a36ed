#!/usr/bin/env python
"""Benchmark of the B200 mode-split step: cell-steps/s of the mixed FP32/FP64 baroclinic step
against the plain FP64 step, on the 2048 x 2048 x 50 irregular domain.

Workload (the reference's large irregular-domain configuration): 2048 x 2048 x 50 sigma layers,
dx = dy = 1 km, seeded land mask of about 30 % (Gaussian-smoothed noise, sigma = 40 cells,
islands kept), depth 5-150 m, stratified T/S with linear EOS, Blumberg-Mellor internal pressure,
P2_PDM / HALFSPLIT advection of momentum and tracers, prescribed parabolic viscosity, closed
boundaries, mode-split ratio M = 20 (dt = 60 s, dtm = 3 s). One STEP = one macro step = 20 micro
steps (integrate_2d) + one integrate_3d. A cell-step is one of the 2048*2048*50 cells (land
included) advanced by one step.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line (rank 0). `--impl reference` times the CPU restatement of the reference's
routines (the oracle, OpenMP over the host cores) on a bounded sample of the same workload.
Multi-GPU runs (torchrun) are weak-scaled replicas: every rank advances its own domain; the
closed-basin step as configured has no inter-rank exchange.
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
WORKLOAD = ("mode-split baroclinic step (20 x integrate_2d + integrate_3d: 2D momentum/sealevel, internal "
            "pressure, 3D momentum with implicit viscosity, P2_PDM advection of u, v, T, S, implicit diffusion), "
            "2048x2048x50 irregular domain, 30% land, depth 5-150 m")
# Algorithmic words (of the 3D fields' precision) per interior cell of each launch of a stage in one
# macro step, each 3D field read or written once counted once; the 2D column heights that the sweeps
# and the diffusion take in place of the 3D height arrays (equidistant sigma) are 1/kmax of a field
# and not counted:
#  * u sweeps: momentum U and V grids (u1: read f, U [+ adv in FP64, where the sum starts from a
#    cleared array; the mixed step's vectorised first sweep starts it itself]; write fi, Di, adv.
#    u2: read f, U, Di, adv; write adv), then the tracer pair (u1: read T, S, U; write T, S, Di.
#    u2: read T, S, U, Di; write T, S, Di);
#  * v sweeps: momentum v1, v2 on both grids (read f, V, Di, adv; write f, Di, adv), tracer pair v1,
#    v2 (read T, S, V, Di; write T, S, Di);
#  * w sweeps: momentum on both grids (read f, ww, hi, adv; write f, hi, adv), tracer pair (read T,
#    S, ww, hi; write T, S, hi);
#  * diffusion: one launch for T and S (read nuh, T, S; write T, S);
# plus, with compensated tracer storage, the FP16 carried errors of T and S read and written by each
# tracer launch (4 x 2 bytes = 2 words of 4 bytes).
STAGE_LAUNCH_WORDS = {"adv_split_u": ([6, 5, 6, 5, 6, 7], [5, 5, 5, 5, 6, 7]),
                      "adv_split_v": ([7, 7, 7, 7, 7, 7], [7, 7, 7, 7, 7, 7]),
                      "adv_split_w": ([7, 7, 7], [7, 7, 7]),
                      "tracer_vdiff": ([5], [5]),
                      "uv_momentum_3d": ([8, 8], [8, 8]),
                      "internal_pressure": ([6], [6])}
LO_WORDS = {"adv_split_u": [0, 0, 0, 0, 2, 2], "adv_split_v": [0, 0, 0, 0, 2, 2], "adv_split_w": [0, 0, 2],
            "tracer_vdiff": [2]}


def stage_words(stage: str, mixed: bool, compensated: bool) -> float:
    """Average algorithmic words per interior cell and launch of a stage of the macro step."""
    w = list(STAGE_LAUNCH_WORDS[stage][1 if mixed else 0])
    if mixed and compensated:
        w = [a + b for a, b in zip(w, LO_WORDS.get(stage, [0] * len(w)))]
    return sum(w) / len(w)
# DRAM bytes (read + write) per interior cell per launch of the FP32 stages, averaged over the
# stage's launches in one macro step: ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum (one
# kernel, up to three launches) on the 1024 x 1024 x 32 case of this workload, scaled per cell
# (v sweeps: four momentum launches at 25.6 and two tracer-pair launches at 34.6; w sweeps: two at
# 21.2 and the pair at 28.2; diffusion: one launch for T and S at 46.5).
TRAFFIC_PER_CELL_F32 = {"adv_split_v": 28.6, "adv_split_w": 23.5, "tracer_vdiff": 46.5}


ERR_FIELDS = ("f3_T", "f3_S", "f3_uu", "f3_vv", "f2_z", "f2_U", "f2_V")


def field_errors(got: dict, ref: dict, az) -> dict:
    """Per field, the largest and the RMS difference of `got` from `ref` over the wet interior cells
    (az == 1; levels 1..kmax of 3D fields), relative to the largest magnitude of the reference field
    and to its range (max - min) there."""
    import torch

    wet2 = az == 1
    out = {}
    for name, b in ref.items():
        a = got[name].double()
        b = b.double()
        if b.dim() == 3:
            m = wet2[None].expand_as(b).clone()
            m[0] = False
        else:
            m = wet2
        bb, d = b[m], (a - b).abs()[m]
        scale = float(bb.abs().max())
        rng = float(bb.max() - bb.min())
        mx, rms = float(d.max()), float(d.pow(2).mean().sqrt())
        out[name[3:]] = {"max": mx / max(scale, 1e-300), "rms": rms / max(scale, 1e-300),
                         "max_range": mx / max(rng, 1e-300), "rms_range": rms / max(rng, 1e-300)}
        del m, bb, d
    torch.cuda.empty_cache()
    return out


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--kmax", type=int, default=50)
    ap.add_argument("--M", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variants", default="fp64,mixed")
    ap.add_argument("--plain-fp32-tracers", dest="compensated", action="store_false",
                    help="mixed step with plain FP32 storage of T and S (no compensation arrays Tlo, Slo)")
    ap.add_argument("--err-steps", type=int, default=200,
                    help="macro steps after which the mixed variant's error against the FP64 variant is stated "
                         "(both variants run on to that step after the timing; the large domain's 200 steps)")
    ap.add_argument("--adj-steps", type=int, default=20, help="tracer steps of the adjoint measurement (0 = skip)")
    ap.add_argument("--adj-every", type=int, default=10, help="checkpoint interval of the adjoint")
    ap.add_argument("--accuracy", type=int, default=0, metavar="STEPS",
                    help="run the mixed-precision accuracy configuration (the 'rotation' recipe: flat 20 m, "
                         "dx = 500 m, closed, solid-body rotation and a temperature anomaly; --nx/--ny/--kmax) for "
                         "STEPS macro steps in FP64 and in the mixed variant and print the per-field errors")
    ap.add_argument("--t-background", type=float, default=0.0,
                    help="accuracy configuration: temperature the tracer blob sits on (0: the tracer-rotation "
                         "configuration's tracer, a unit blob plus noise on zero)")
    ap.add_argument("--configs", action="store_true",
                    help="time the smaller configurations: the 128x128x20 tracer rotation (200 steps) and the "
                         "512x512x30 tidal shelf (100 macro steps), GPU FP64 / mixed and the CPU oracle on the "
                         "host cores (a 5-macro-step sample for the shelf); one JSON line")
    ap.add_argument("--cpu-sizes", default="", metavar="N,N,...",
                    help="time the CPU oracle (the reported CPU baseline) on the islands recipe at each NxN size "
                         "(kmax and M of the workload) and print its rate per size; one JSON line")
    ap.add_argument("--tile-sweeps", action="store_true",
                    help="use the shared-memory tile kernels for every horizontal sweep (comparison)")
    ap.add_argument("--tracer-adjoint", action="store_true",
                    help="time only the checkpointed tracer gradient on the tracer-adjoint configuration "
                         "(random divergence-free flow, SUPERBEE, implicit diffusion; --nx/--ny/--kmax, "
                         "--adj-steps, --adj-every) in FP64 and FP32 and print one JSON line")
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
        self.out = ""

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
        return False

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = sorted(v for v in (num(r[1]) for r in rows) if v is not None)
        mx = max((v for v in (num(r[2]) for r in rows) if v is not None), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def reduce_max(x: float, world: int, device: str) -> float:
    """The largest of the ranks' values (the job's time is its slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(cells_per_rank: int, steps: int, world: int, ms_max: float) -> float:
    """cell-steps/s of the whole job: every rank advances its own domain (weak scaling)."""
    return world * cells_per_rank * steps / (ms_max / 1e3)


def dist_setup():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def oracle_sample(nx, ny, kmax, M):
    from code_b200 import state as S

    return S.baroclinic_case(nx=nx, ny=ny, kmax=kmax, recipe="islands", land=0.3, M=M, dt3=60.0, seed=6)


def cpu_build():
    """Select the oracle build tuned for this host's CPU (-march=native, built here with the
    system g++), falling back to the portable build; returns the flags of the build in use."""
    import oracle

    oracle.use_native_build()
    return oracle.BUILD_FLAGS[oracle.variant]


def run_reference(args, world, rank):
    """CPU restatement (oracle) on a bounded sample of the workload, all host threads."""
    if rank != 0:
        return
    import oracle

    flags = cpu_build()

    # a 512x512 sample per step (the per-cell rate at 512x512 is within 3% of the rate the larger
    # samples level off at, and a step takes ~1.6 s on 16 host cores)
    snx = min(args.nx, 512)
    sny = min(args.ny, 512)
    c = oracle_sample(snx, sny, args.kmax, args.M)
    M = args.M
    n = 1
    for _ in range(args.warmup):
        oracle.bc_steps(c, n, M)
        n += M
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.bc_steps(c, n, M)
        n += M
    el = time.perf_counter() - t0
    cells = snx * sny * args.kmax
    v = cells * args.steps / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "nx": args.nx, "ny": args.ny, "kmax": args.kmax, "M": M,
                   "sample": f"{snx}x{sny}x{args.kmax} islands domain per step"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "build": flags,
                         "sample": f"oracle FP64 mode-split step on {snx}x{sny}x{args.kmax}, {args.steps} macro steps "
                                   f"after {args.warmup} warm-up"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def cpu_baseline_sample(args):
    import oracle

    flags = cpu_build()
    # the 1024x1024 sample: the oracle's per-cell rate has levelled off at that size
    snx, sny = min(args.nx, 1024), min(args.ny, 1024)
    c = oracle_sample(snx, sny, args.kmax, args.M)
    oracle.bc_steps(c, 1, args.M)
    n, steps, t0 = 1 + args.M, 0, time.perf_counter()
    while True:
        oracle.bc_steps(c, n, args.M)
        n += args.M
        steps += 1
        el = time.perf_counter() - t0
        if el > 10.0 or steps >= 20:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": snx * sny * args.kmax * steps / el, "unit": UNIT, "cores": cores, "kind": "port", "build": flags,
            "sample": f"oracle FP64 mode-split step on {snx}x{sny}x{args.kmax} (islands), {steps} macro steps "
                      f"({el:.1f} s)"}


def run_cpu_sizes(args):
    """Per-cell rate of the CPU oracle (the timed baseline) against the sample size: the islands
    recipe at each size of --cpu-sizes (kmax and M of the workload), one warm-up macro step, then
    timed macro steps for at least 10 s (at least one)."""
    import oracle

    flags = cpu_build()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    rows = []
    for n in (int(x) for x in args.cpu_sizes.split(",")):
        c = oracle_sample(n, n, args.kmax, args.M)
        oracle.bc_steps(c, 1, args.M)
        k, t0, el = 1 + args.M, time.perf_counter(), 0.0
        steps = 0
        while steps < 1 or el < 10.0:
            oracle.bc_steps(c, k, args.M)
            k += args.M
            steps += 1
            el = time.perf_counter() - t0
        rows.append({"size": f"{n}x{n}x{args.kmax}", "cells": n * n * args.kmax, "macro_steps": steps,
                     "s_per_step": el / steps, "value": n * n * args.kmax * steps / el})
        del c
    print(json.dumps({"cpu_oracle_rate_by_size": rows, "unit": UNIT, "cores": cores, "build": flags,
                      "workload": f"islands recipe, kmax = {args.kmax}, M = {args.M}"}), flush=True)


def run_tracer_adjoint(args):
    """The tracer-adjoint configuration (256 x 256 x 30, flat 30 m, dx = 500 m, 8-mode random
    streamfunction flow with max 0.5 m/s, SUPERBEE HALFSPLIT, nuh = 1e-4, J = tracer content of the
    central 32 x 32 box): device time of the forward pass (with checkpoints) and of the reverse pass
    of getm_tracer_gradient, FP64 and FP32."""
    import numpy as np
    import torch

    from code_b200 import cases
    from code_b200.getm import Context

    c = cases.streamfunction_flow(nx=args.nx, ny=args.ny, kmax=args.kmax, dt=300.0, seed=4)
    c.par.update(cnpar=1.0, avmol=0.0)
    p = c.par
    w = cases.box_weights(c, box=min(32, args.nx, args.ny))
    ctx = Context(c.grid)
    ctx.init_advection(*[torch.from_numpy(m).cuda() for m in c.masks()])
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    out = {"workload": f"tracer adjoint: {args.nx}x{args.ny}x{args.kmax}, {args.adj_steps} steps, checkpoint every "
                       f"{args.adj_every}, SUPERBEE HALFSPLIT + implicit diffusion", "results": {}}
    for name, dt in (("f64", torch.float64), ("f32", torch.float32)):
        t = [torch.from_numpy(c[n]).cuda().to(dt) for n in names]
        runs = []
        for rep in range(max(2, args.warmup)):
            f = torch.from_numpy(c["f"]).cuda().to(dt)
            fbar = torch.from_numpy(w).cuda().to(dt)
            nubar = torch.zeros_like(fbar)
            torch.cuda.synchronize()
            runs.append(ctx.tracer_gradient(args.adj_steps, args.adj_every, p["dt"], f, *t, p["split"], p["hscheme"],
                                            p["vscheme"], p["AH"], p["cnpar"], p["avmol"], fbar, nubar))
        ms_f, ms_r = runs[-1]
        out["results"][name] = {"ms_forward": ms_f, "ms_reverse": ms_r, "adjoint_fwd_ratio": ms_r / ms_f,
                                "grad_norm": float(fbar.double().norm())}
    ctx.close()
    print(json.dumps(out), flush=True)


def run_configs(args):
    """Device and host throughput of the tracer-rotation and tidal-shelf configurations."""
    import numpy as np
    import torch

    import oracle
    from code_b200 import cases
    from code_b200 import state as S
    from code_b200.getm import BcDevice, Context

    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    out = {"cores": cores, "unit": UNIT}
    # tracer rotation: 128 x 128 x 20, SUPERBEE HALFSPLIT, implicit diffusion, 200 steps
    c = cases.tracer_rotation()
    p = c.par
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    cells = c.grid.nx * c.grid.ny * c.grid.kmax
    res = {}
    for key, dt in (("gpu_fp64", torch.float64), ("gpu_fp32", torch.float32)):
        ctx = Context(c.grid)
        ctx.init_advection(*[torch.from_numpy(m).cuda() for m in c.masks()])
        f = torch.from_numpy(c["f"]).cuda().to(dt)
        t = [torch.from_numpy(c[n]).cuda().to(dt) for n in names]
        for _ in range(3):
            ctx.tracer_step(p["dt"], f.clone(), *t, p["split"], p["hscheme"], p["vscheme"], p["AH"], p["cnpar"],
                            p["avmol"])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(200):
            ctx.tracer_step(p["dt"], f, *t, p["split"], p["hscheme"], p["vscheme"], p["AH"], p["cnpar"], p["avmol"])
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[key] = {"ms_per_step": ms / 200, "value": cells * 200 / (ms / 1e3)}
        ctx.close()
    o = oracle.Oracle(c.grid)
    of = c["f"].copy()
    t0 = time.perf_counter()
    o.tracer_steps(c.masks(), 200, p["dt"], of, *[c[n] for n in names], p["split"], p["hscheme"], p["vscheme"],
                   p["AH"], p["cnpar"], p["avmol"])
    el = time.perf_counter() - t0
    res["cpu_oracle_fp64"] = {"ms_per_step": el * 1e3 / 200, "value": cells * 200 / el}
    out["tracer_rotation_128x128x20"] = res
    # tidal shelf: 512 x 512 x 30, M = 20, M2 tide (1 m) on the western boundary
    g = S.Grid(512, 512, 30, 1000.0, 1000.0)
    b = S.OpenBoundaries(west=[(g.imin, g.jmin, g.jmax, S.CLAMPED)], ramp=40, amp=1.0, period=44712.0)
    c2 = S.baroclinic_case(nx=512, ny=512, kmax=30, recipe="shelf", M=20, dt3=60.0, seed=3, bdy=b)
    cells = 512 * 512 * 30
    res = {}
    for key, dt3 in (("gpu_fp64", torch.float64), ("gpu_mixed", torch.float32)):
        cc = c2.copy(dtype3=np.float32 if dt3 == torch.float32 else None)
        ctx = Context(cc.grid)
        ctx.init_advection(*[torch.from_numpy(m).cuda() for m in cc.masks()])
        ctx.set_open_boundaries(cc.bdy)
        st = BcDevice(cc, dtype3=dt3)
        ctx.time_loop(st, 1, 20 * 3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.time_loop(st, 61, 20 * 100)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[key] = {"ms_per_step": ms / 100, "value": cells * 100 / (ms / 1e3)}
        ctx.close()
        del st
    cs = c2.copy()
    t0 = time.perf_counter()
    oracle.bc_steps(cs, 1, 20 * 5)
    el = time.perf_counter() - t0
    res["cpu_oracle_fp64"] = {"ms_per_step": el * 1e3 / 5, "value": cells * 5 / el, "sample": "5 macro steps"}
    out["tidal_shelf_512x512x30"] = res
    print(json.dumps(out), flush=True)


def run_accuracy(args):
    """Mixed variant against the FP64 variant after args.accuracy macro steps: per field, the largest
    and the RMS difference relative to the largest magnitude of the FP64 field."""
    import numpy as np
    import torch

    from code_b200 import state as S
    from code_b200.getm import BcDevice, Context

    c = S.baroclinic_case(nx=args.nx, ny=args.ny, kmax=args.kmax, recipe="rotation", dx=500.0, M=args.M, dt3=60.0,
                          seed=3, t_background=args.t_background, t_noise=1e-3)
    res = {}
    t0 = time.time()
    for key, dt in (("fp64", torch.float64), ("mixed", torch.float32)):
        ctx = Context(c.grid)
        ctx.init_advection(*[torch.from_numpy(m).cuda() for m in c.masks()])
        st = BcDevice(c, dtype3=dt, compensated=args.compensated)
        ctx.time_loop(st, 1, args.M * args.accuracy)
        torch.cuda.synchronize()
        res[key] = {n: st.t[n].clone() for n in ERR_FIELDS}
        az = st.t["az"]
        ctx.close()
        del st
    err = field_errors(res["mixed"], res["fp64"], az)
    print(json.dumps({"workload": f"mixed-precision accuracy: rotation recipe {args.nx}x{args.ny}x{args.kmax}, "
                                  f"M = {args.M}, {args.accuracy} macro steps, tracer: Gaussian blob of amplitude 1 "
                                  f"plus uniform noise of 1e-3 on {args.t_background} C; tracer storage "
                                  f"{'FP32 with compensation' if args.compensated else 'FP32'}",
                      "relative_to": "max: max |field| of the FP64 run; range: its max - min; wet interior cells",
                      "errors": err, "wall_s": time.time() - t0}), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.tile_sweeps and args.impl != "reference":
        from code_b200 import getm as G

        G.set_vector_sweeps(False)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.tracer_adjoint:
        if rank == 0:
            run_tracer_adjoint(args)
        return
    if args.accuracy > 0:
        if rank == 0:
            run_accuracy(args)
        return
    if args.configs:
        if rank == 0:
            run_configs(args)
        return
    if args.cpu_sizes:
        if rank == 0:
            run_cpu_sizes(args)
        return
    import torch
    import torch.distributed as dist

    from code_b200 import state as S
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
        return reduce_max(x, world, "cuda")

    M = args.M
    cells = args.nx * args.ny * args.kmax
    variants = {}
    wanted = args.variants.split(",")
    for key, dt3 in (("fp64", torch.float64), ("mixed", torch.float32)):
        if key not in wanted:
            continue
        g, st = S.baroclinic_case_device(args.nx, args.ny, args.kmax, recipe="islands", land=0.3, M=M, dt3=60.0,
                                         seed=6 + rank, dtype3=dt3, compensated=args.compensated)
        ctx = Context(g, stream)
        ctx.init_advection(*st.masks())
        variants[key] = dict(g=g, st=st, ctx=ctx, n=1)

    def macro_step(key):
        v = variants[key]
        v["ctx"].time_loop(v["st"], v["n"], M)
        v["n"] += M

    res = {}
    clocks = None
    for key in variants:
        for _ in range(args.warmup):
            macro_step(key)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as cs:
            e0.record(stream)
            for _ in range(args.steps):
                macro_step(key)
            e1.record(stream)
            barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        res[key] = {"ms": ms, "value": whole_job_value(cells, args.steps, world, ms)}
        if key == "mixed" or clocks is None:
            clocks = cs.summary()
    # stated error of the mixed variant against the FP64 run after the same number of steps
    err = None
    if "fp64" in variants and "mixed" in variants and variants["fp64"]["n"] == variants["mixed"]["n"]:
        # both variants on to the stated number of macro steps (outside the timed region)
        while (variants["fp64"]["n"] - 1) // M < args.err_steps:
            macro_step("fp64")
            macro_step("mixed")
        torch.cuda.synchronize()
        err = {"steps": (variants["fp64"]["n"] - 1) // M,
               "relative_to": "max: max |field| of the FP64 run; range: its max - min; wet interior cells"}
        err.update(field_errors({n: variants["mixed"]["st"].t[n] for n in ERR_FIELDS},
                                {n: variants["fp64"]["st"].t[n] for n in ERR_FIELDS}, variants["fp64"]["st"].t["az"]))
    head = "mixed" if "mixed" in variants else "fp64"
    v = variants[head]
    # per-stage device timers over K more steps of the headline variant (dominant kernel roofline)
    v["ctx"].timers(enable=True, reset=True)
    for _ in range(args.steps):
        macro_step(head)
    torch.cuda.synchronize()
    tim = v["ctx"].timers(enable=False, reset=True)
    launches = sum(n for _, n in tim.values())
    # the same per-stage breakdown of the plain FP64 step, for the comparison
    tim64 = None
    if head == "mixed" and "fp64" in variants:
        c64 = variants["fp64"]["ctx"]
        c64.timers(enable=True, reset=True)
        for _ in range(args.steps):
            macro_step("fp64")
        torch.cuda.synchronize()
        tim64 = c64.timers(enable=False, reset=True)
    timed = {k: t for k, t in tim.items() if k in STAGE_LAUNCH_WORDS}
    top_name, (top_ms, top_n) = max(timed.items(), key=lambda kv: kv[1][0])
    wb = 4 if head == "mixed" else 8
    alg_bytes = stage_words(top_name, head == "mixed", args.compensated) * cells * wb
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (top_ms / top_n / 1e3) / 1e9
    # whole-step algorithmic bytes (3D: read+write uu, vv, T, S; 2D: 17 FP64 words per column per micro step)
    step_bytes = (8 * wb) * cells + 17 * 8 * args.nx * args.ny * M
    # end to end through the C ABI with host buffers: per step the 2D forcing (tausx, tausy, airp) is
    # uploaded from pinned host memory and the new elevation z read back. The copies run on a copy
    # stream, overlapped with the steps as a host driving the library would pipeline them: step
    # n+1's forcing goes up into device staging buffers while step n computes (the step then takes
    # it with device copies), and step n's elevation comes down from a device copy of it while
    # step n+1 computes; the timed region ends when the last elevation is on the host.
    st = v["st"]
    forcing = ("tausx", "tausy", "airp")
    hf = {n: torch.empty_like(st.t["f2_" + n], device="cpu").pin_memory() for n in forcing + ("z",)}
    for n in forcing:
        hf[n].copy_(st.t["f2_" + n])
    up = {n: torch.empty_like(st.t["f2_" + n]) for n in forcing}
    zdev = torch.empty_like(st.t["f2_z"])
    cstream = torch.cuda.Stream()
    barrier()
    k2 = max(3, args.steps // 2)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cstream.wait_event(e0)

    def upload():
        with torch.cuda.stream(cstream):
            for n in forcing:
                up[n].copy_(hf[n], non_blocking=True)
            return cstream.record_event()

    up_done, down_done = upload(), None
    for it in range(k2):
        stream.wait_event(up_done)
        for n in forcing:
            st.t["f2_" + n].copy_(up[n])
        taken = stream.record_event()
        if it + 1 < k2:
            cstream.wait_event(taken)
            up_done = upload()
        macro_step(head)
        if down_done is not None:
            stream.wait_event(down_done)  # zdev is free again
        zdev.copy_(st.t["f2_z"])
        z_ready = stream.record_event()
        with torch.cuda.stream(cstream):
            cstream.wait_event(z_ready)
            hf["z"].copy_(zdev, non_blocking=True)
            down_done = cstream.record_event()
    stream.wait_event(down_done)
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    n2b = st.t["f2_z"].numel() * 8
    # adjoint of the tracer subsystem on the headline state: gradient of the salinity content of a
    # central 512 x 512 column block after adj_steps tracer steps (advection + implicit diffusion,
    # velocities, layer heights and nuh of the current state), checkpointed every adj_every steps;
    # ratio = device time of the reverse pass (recomputation included) / forward pass
    adj = None
    if args.adj_steps > 0:
        t3, pd, pi = st.t, st.pd, st.pi
        fs = t3["f3_S"].clone()
        wgt = torch.zeros_like(fs)
        g = v["g"]
        b = min(512, args.nx, args.ny)
        j0, i0 = 2 + (args.ny - b) // 2, 2 + (args.nx - b) // 2
        wgt[1:, j0:j0 + b, i0:i0 + b] = t3["f3_hn"][1:, j0:j0 + b, i0:i0 + b] / g.ard1
        wgt *= (t3["az"] == 1).to(wgt.dtype)[None]
        nubar = torch.zeros_like(fs)
        args3 = [t3["f3_" + n] for n in ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")]
        adj_ms = []
        for rep in range(2):  # the first call allocates the checkpoints and tapes
            f = fs.clone()
            fbar = wgt.clone()
            nubar.zero_()
            barrier()
            ms_f, ms_r = v["ctx"].tracer_gradient(args.adj_steps, args.adj_every, pd["dt"], f, *args3,
                                                  pi["salt_adv_split"], pi["salt_adv_hor"], pi["salt_adv_ver"],
                                                  pd["salt_AH"], pd["cnpar"], pd["avmols"], fbar, nubar)
            adj_ms.append((max_over_ranks(ms_f), max_over_ranks(ms_r)))
        ms_f, ms_r = adj_ms[-1]
        adj = {"steps": args.adj_steps, "checkpoint_every": args.adj_every, "field": "S",
               "dtype": "f32" if fs.dtype == torch.float32 else "f64", "ms_forward": ms_f, "ms_reverse": ms_r,
               "objective": f"salinity content of the central {b}x{b} column block"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_sample(args)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}
    if rank == 0:
        out = {
            "metric": METRIC, "value": res[head]["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res[head]["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if head == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "nx": args.nx, "ny": args.ny, "kmax": args.kmax, "M": M,
                       "l2": "inputs larger than L2 (one FP32 3D field 0.86 GB)", "parallelism": f"replicas x{world}",
                       "tracer_storage": ("FP32 with compensation (T + Tlo, S + Slo)" if args.compensated
                                          else "FP32")},
            "plain_fp64": ({"value": res["fp64"]["value"], "ms_per_step": res["fp64"]["ms"] / args.steps}
                           if "fp64" in res else None),
            "mixed_over_fp64": (res["mixed"]["value"] / res["fp64"]["value"]) if len(res) == 2 else None,
            "err_vs_fp64": err,
            "adjoint_fwd_ratio": (adj["ms_reverse"] / adj["ms_forward"]) if adj else None,
            "adjoint": adj,
            "gpu_launches": launches,
            "stage_ms_per_step": {k: t[0] / args.steps for k, t in tim.items()},
            "stage_ms_per_step_fp64": ({k: t[0] / args.steps for k, t in tim64.items()} if tim64 else None),
            "roofline": {"bound": "hbm", "kernel": top_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (TRAFFIC_PER_CELL_F32[top_name] * cells
                                     if head == "mixed" and top_name in TRAFFIC_PER_CELL_F32 else None),
                         "alg_bytes_per_launch": alg_bytes,
                         "step_alg_bytes": step_bytes,
                         "step_frac": step_bytes / (res[head]["ms"] / args.steps / 1e3) / 1e9 / peak},
            "e2e": {"value": world * cells * k2 / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 3 * n2b,
                    "d2h_bytes_per_step": n2b},
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out), flush=True)
    for key in variants:
        variants[key]["ctx"].close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
