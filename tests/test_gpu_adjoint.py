"""Adjoint of the tracer step on the GPU, through the C ABI.

Checks (FP64 unless stated):
  * the recording forward step advances the tracer exactly like getm_tracer_step;
  * one adjoint step against the oracle's tangent-linear step (dual numbers):
    <fbar0, df> + <nubar, dnuh> = <w, tangent(df, dnuh)> for every split scheme, to 1e-10;
  * the checkpointed multi-step gradient against the tangent-linear oracle (1e-9) and against the
    step-by-step adjoint (bit for bit);
  * the gradient against central finite differences of the GPU forward run (1e-4): dJ/df0 and
    dJ/dnuh with the linear P2 scheme, and dJ/df0 on 64 directions in the tracer-adjoint
    configuration (256 x 256 x 30, SUPERBEE, 50 steps);
  * the FP32 gradient against the FP64 tangent (1e-4 with P2; 1e-3 with SUPERBEE, see the test).
"""
import numpy as np
import pytest

import oracle
from code_b200 import cases
from code_b200 import getm as G
from helpers import dev, host, make_ctx

pytestmark = pytest.mark.gpu

NAMES = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn")
SCHEMES = {"UPSTREAM": 1, "P2": 3, "SUPERBEE": 4, "MUSCL": 5, "P2_PDM": 6}


def _dev_fields(c, dtype=None):
    import torch

    t = {n: dev(c[n]) for n in NAMES + ("nuh",)}
    if dtype is not None:
        t = {n: v.to(dtype) for n, v in t.items()}
    return t


def _steps(ctx, c, t, f, nsteps, hs, vs):
    p = c.par
    for _ in range(nsteps):
        ctx.tracer_step(p["dt"], f, *[t[n] for n in NAMES], t["nuh"], 2, hs, vs, p["AH"], p["cnpar"], p["avmol"])


def test_record_step_equals_plain_step():
    import torch

    c = cases.random_case(nx=37, ny=29, kmax=9, seed=3)
    c.par.update(AH=0.0, cnpar=0.9, avmol=1e-6)
    ctx, m = make_ctx(c)
    for dtype in (torch.float64, torch.float32):
        t = _dev_fields(c, dtype)
        f1 = dev(c["f"]).to(dtype)
        f2 = f1.clone()
        tape = ctx.tape(dtype)
        _steps(ctx, c, t, f1, 1, 6, 6)
        ctx.tracer_step_record(c.par["dt"], f2, *[t[n] for n in NAMES], t["nuh"], 2, 6, 6, 0.0, 0.9, 1e-6, tape)
        torch.cuda.synchronize()
        if dtype == torch.float64:
            assert torch.equal(f1, f2)
        else:
            assert torch.allclose(f1, f2, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("scheme", list(SCHEMES))
@pytest.mark.parametrize("AH", [0.0, 5.0])
def test_adjoint_step_vs_tangent(scheme, AH):
    import torch

    hs = SCHEMES[scheme]
    c = cases.random_case(nx=33, ny=27, kmax=8, seed=11)
    p = c.par
    p.update(AH=AH, cnpar=0.9, avmol=1e-6, split=2, hscheme=hs, vscheme=hs)
    o = oracle.Oracle(c.grid)
    ctx, m = make_ctx(c)
    t = _dev_fields(c)
    rng = np.random.default_rng(7)
    w = rng.normal(size=c["f"].shape)
    df = rng.normal(size=c["f"].shape)
    dnuh = rng.normal(size=c["f"].shape) * 1e-3
    # tangent on the CPU
    fo, dfo = c["f"].copy(), df.copy()
    o.tracer_steps_tl(c.masks(), 1, p["dt"], fo, dfo, *[c[n] for n in NAMES], c["nuh"], dnuh, 2, hs, hs, AH,
                      p["cnpar"], p["avmol"])
    tl = float(np.sum(w * dfo))
    # adjoint on the GPU
    f = dev(c["f"])
    tape = ctx.tape(torch.float64)
    ctx.tracer_step_record(p["dt"], f, *[t[n] for n in NAMES], t["nuh"], 2, hs, hs, AH, p["cnpar"], p["avmol"],
                           tape)
    assert np.array_equal(host(f), fo)  # the tangent's values are the plain FP64 step
    fbar = dev(w)
    nubar = torch.zeros_like(fbar)
    ctx.tracer_step_adjoint(p["dt"], fbar, nubar, *[t[n] for n in NAMES], t["nuh"], 2, hs, hs, AH, p["cnpar"],
                            p["avmol"], tape)
    ad = float(np.sum(host(fbar) * df) + np.sum(host(nubar) * dnuh))
    assert abs(ad - tl) <= 1e-10 * (abs(tl) + 1e-300), (ad, tl)


def _flow(nx=48, ny=40, kmax=8):
    c = cases.streamfunction_flow(nx=nx, ny=ny, kmax=kmax, dt=300.0, seed=4)
    c.par.update(cnpar=0.9, avmol=1e-6)
    return c


def _gradient(ctx, c, t, nsteps, every, w, dtype=None):
    import torch

    p = c.par
    f = dev(c["f"]) if dtype is None else dev(c["f"]).to(dtype)
    fbar = dev(w) if dtype is None else dev(w).to(dtype)
    nubar = torch.zeros_like(fbar)
    ms = ctx.tracer_gradient(nsteps, every, p["dt"], f, *[t[n] for n in NAMES], t["nuh"], 2, p["hscheme"],
                             p["vscheme"], p["AH"], p["cnpar"], p["avmol"], fbar, nubar)
    return f, fbar, nubar, ms


def test_gradient_vs_tangent_and_stepwise():
    import torch

    c = _flow()
    p = c.par
    o = oracle.Oracle(c.grid)
    ctx, m = make_ctx(c)
    t = _dev_fields(c)
    w = cases.box_weights(c, box=16)
    nsteps, every = 12, 5
    f, fbar, nubar, _ = _gradient(ctx, c, t, nsteps, every, w)
    # final state = plain forward
    fp = dev(c["f"])
    _steps(ctx, c, t, fp, nsteps, p["hscheme"], p["vscheme"])
    assert torch.equal(f, fp)
    # step-by-step adjoint with every tape kept
    fs = dev(c["f"])
    tapes = []
    for _ in range(nsteps):
        tp = ctx.tape(torch.float64)
        ctx.tracer_step_record(p["dt"], fs, *[t[n] for n in NAMES], t["nuh"], 2, p["hscheme"], p["vscheme"],
                               p["AH"], p["cnpar"], p["avmol"], tp)
        tapes.append(tp)
    gb = dev(w)
    nb = torch.zeros_like(gb)
    for tp in reversed(tapes):
        ctx.tracer_step_adjoint(p["dt"], gb, nb, *[t[n] for n in NAMES], t["nuh"], 2, p["hscheme"], p["vscheme"],
                                p["AH"], p["cnpar"], p["avmol"], tp)
    assert torch.equal(gb, fbar) and torch.equal(nb, nubar)
    # tangent-linear oracle on four directions
    rng = np.random.default_rng(5)
    G, NB = host(fbar), host(nubar)
    for q in range(4):
        df = rng.normal(size=c["f"].shape) * (c["az"] >= 1)[None]
        dnuh = rng.normal(size=c["f"].shape) * 1e-5 if q % 2 else None
        fo, dfo = c["f"].copy(), df.copy()
        o.tracer_steps_tl(c.masks(), nsteps, p["dt"], fo, dfo, *[c[n] for n in NAMES], c["nuh"], dnuh, 2,
                          p["hscheme"], p["vscheme"], p["AH"], p["cnpar"], p["avmol"])
        tl = float(np.sum(w * dfo))
        ad = float(np.sum(G * df) + (np.sum(NB * dnuh) if dnuh is not None else 0.0))
        assert abs(ad - tl) <= 1e-9 * abs(tl), (q, ad, tl)


def _fd_errors(c, nsteps, every, box, dirs, eps_f, eps_nu):
    """Relative differences between the directional derivatives of the checkpointed gradient and
    central differences of the GPU forward run; dirs = sequence of "f" / "nuh". J(+) - J(-) is
    taken as sum(w * (f+ - f-)) so that the two large sums do not cancel."""
    import torch

    p = c.par
    ctx, m = make_ctx(c)
    t = _dev_fields(c)
    w = cases.box_weights(c, box=box)
    wt = dev(w)
    _, fbar, nubar, _ = _gradient(ctx, c, t, nsteps, every, w)
    rng = np.random.default_rng(5)
    wet = torch.from_numpy((c["az"] >= 1)[None].astype(np.float64)).cuda()

    def run(f0, nuh):
        f = f0.clone()
        for _ in range(nsteps):
            ctx.tracer_step(p["dt"], f, *[t[n] for n in NAMES], nuh, 2, p["hscheme"], p["vscheme"], p["AH"],
                            p["cnpar"], p["avmol"])
        return f

    f0 = dev(c["f"])
    errs = []
    for which in dirs:
        d = torch.from_numpy(rng.normal(size=c["f"].shape)).cuda() * wet
        if which == "f":
            fd = float(torch.sum(wt * (run(f0 + eps_f * d, t["nuh"]) - run(f0 - eps_f * d, t["nuh"])))) / (2 * eps_f)
            ad = float(torch.sum(fbar * d))
        else:
            d = d * t["nuh"]  # relative perturbation of the diffusivity
            fd = float(torch.sum(wt * (run(f0, t["nuh"] + eps_nu * d) - run(f0, t["nuh"] - eps_nu * d)))) / (2 * eps_nu)
            ad = float(torch.sum(nubar * d))
        errs.append(abs(ad - fd) / abs(fd))
    return np.array(errs)


def test_gradient_vs_finite_differences_p2():
    """P2 (the unlimited, linear scheme), vertically sheared flow, stratified tracer: both dJ/df0
    and dJ/dnuh agree with central differences to 1e-4 (about 1e-7 obtained)."""
    c = cases.streamfunction_flow(nx=64, ny=64, kmax=10, dt=300.0, seed=4, vertical=0.5, shear=1.0)
    c.par.update(cnpar=0.9, avmol=1e-6, hscheme=3, vscheme=3)
    errs = _fd_errors(c, 20, 10, 32, ["f", "nuh"] * 4, eps_f=1e-6, eps_nu=1e-3)
    assert errs.max() <= 1e-4, errs


def test_gradient_tracer_adjoint_configuration_fd():
    """The tracer-adjoint configuration: 256 x 256 x 30, flat 30 m, dx = 500 m, random
    divergence-free flow (8 modes, max 0.5 m/s), SUPERBEE + implicit diffusion (nuh = 1e-4),
    50 steps checkpointed every 10, J = tracer content of the central 32 x 32 box. dJ/df0 against
    central differences on 64 seeded random directions: median <= 1e-5, at least 60 of the 64
    within 1e-4, all within 1e-3. TVD limiters are piecewise linear in the tracer; with 1e7 faces per step some faces
    always sit within the perturbation of a kink, and a secant that crosses one measures a slightly
    different map (the frozen-branch gradient itself is checked exactly against the tangent-linear
    model above). Directions in nuh move the limiter ratio of every face at once; for SUPERBEE
    they are checked against the tangent-linear model instead."""
    c = cases.streamfunction_flow(nx=256, ny=256, kmax=30, dt=300.0, seed=4)
    c.par.update(cnpar=1.0, avmol=0.0)
    errs = _fd_errors(c, 50, 10, 32, ["f"] * 64, eps_f=1e-9, eps_nu=None)
    print(f"64 directions: median {np.median(errs):.1e}, max {errs.max():.1e}, "
          f"{int((errs > 1e-4).sum())} above 1e-4")
    assert np.median(errs) <= 1e-5 and (errs > 1e-4).sum() <= 4 and errs.max() <= 1e-3, errs


def _fd_sweep(c, nsteps, every, box, which, eps_list, ndirs=64):
    """{eps: (relative differences, limiter-branch flips)} of the directional derivatives of the
    checkpointed gradient against central differences of the GPU forward run, on the same ndirs
    seeded directions for every eps; which = "f" (initial tracer) or "nuh" (relative perturbation
    of the diffusivity). The two forward runs of a difference record their limiter branches
    (getm_tracer_step_record, the same bits as getm_tracer_step); flips = the number of faces and
    steps at which the + and - runs took different branches, i.e. at which the secant crosses a
    kink of the piecewise-linear step."""
    import torch

    p = c.par
    ctx, m = make_ctx(c)
    t = _dev_fields(c)
    w = cases.box_weights(c, box=box)
    wt = dev(w)
    _, fbar, nubar, _ = _gradient(ctx, c, t, nsteps, every, w)
    rng = np.random.default_rng(11 if which == "f" else 12)
    wet = torch.from_numpy((c["az"] >= 1)[None].astype(np.float64)).cuda()
    tapes = [ctx.tape(torch.float64), ctx.tape(torch.float64)]
    for tp in tapes:
        tp[0].zero_()

    def run(f0, nuh, tp, codes):
        f = f0.clone()
        for q in range(nsteps):
            ctx.tracer_step_record(p["dt"], f, *[t[n] for n in NAMES], nuh, 2, p["hscheme"], p["vscheme"], p["AH"],
                                   p["cnpar"], p["avmol"], tp)
            codes[q].copy_(tp[0])
        return f

    codes = [[torch.empty_like(tapes[0][0]) for _ in range(nsteps)] for _ in range(2)]
    f0 = dev(c["f"])
    dirs = [torch.from_numpy(rng.normal(size=c["f"].shape)).cuda() * wet for _ in range(ndirs)]
    out = {}
    for eps in eps_list:
        errs, flips = [], []
        for d in dirs:
            if which == "f":
                fp = run(f0 + eps * d, t["nuh"], tapes[0], codes[0])
                fm = run(f0 - eps * d, t["nuh"], tapes[1], codes[1])
                ad = float(torch.sum(fbar * d))
            else:
                dn = d * t["nuh"]
                fp = run(f0, t["nuh"] + eps * dn, tapes[0], codes[0])
                fm = run(f0, t["nuh"] - eps * dn, tapes[1], codes[1])
                ad = float(torch.sum(nubar * dn))
            fd = float(torch.sum(wt * (fp - fm))) / (2 * eps)
            errs.append(abs(ad - fd) / abs(fd))
            flips.append(int(sum(int(torch.count_nonzero(a != b)) for a, b in zip(codes[0], codes[1]))))
        out[eps] = (np.array(errs), np.array(flips))
    return out


def _report(which, res):
    for eps, (e, fl) in res.items():
        calm = e[fl == 0]
        print(f"d{which} eps {eps:.0e}: median {np.median(e):.1e}, max {e.max():.1e}, "
              f"{int((e <= 1e-4).sum())}/{len(e)} within 1e-4; {len(calm)} directions without branch flips"
              + (f" (max {calm.max():.1e})" if len(calm) else "") + f"; flips per direction median {np.median(fl):.0f}")


@pytest.mark.parametrize("which,eps_list", [("f", (1e-7, 1e-9, 1e-11)), ("nuh", (1e-2, 1e-4, 1e-6))])
def test_tracer_adjoint_configuration_fd_sweep(which, eps_list):
    """Both gradients of the tracer-adjoint configuration (256 x 256 x 30, SUPERBEE, 50 steps,
    checkpoint every 10) against central differences on 64 seeded directions, for three step sizes
    each: dJ/df0 (absolute steps on a tracer of range ~1) and dJ/dnuh (relative perturbations of
    the diffusivity). Prints the median, the maximum, the share within 1e-4 and the limiter-branch
    flips per direction. The step is piecewise linear in the tracer (SUPERBEE's branches) and the
    gradient is that of the branches the forward run took, exactly (checked against the
    tangent-linear model above); every secant here crosses kinks (no direction is flip-free, even
    at 1e-11). In this configuration the flow is the same in every layer and the tracer's vertical
    structure is its 1e-3 noise, so the diffusion only moves tracer within columns and J depends on
    nuh only through the limiters (with a linear scheme dJ/dnuh is exactly zero: see the next
    test): dJ/dnuh is the derivative of the branch pattern itself, which the secants measure to a
    median of about 1e-3. Bounds at the best step size: dJ/df0 median 1e-5 and 56 of 64 within
    1e-4; dJ/dnuh median 2e-3."""
    c = cases.streamfunction_flow(nx=256, ny=256, kmax=30, dt=300.0, seed=4)
    c.par.update(cnpar=1.0, avmol=0.0)
    res = _fd_sweep(c, 50, 10, 32, which, eps_list)
    _report(which, res)
    best = max((e for e, _ in res.values()), key=lambda e: ((e <= 1e-4).sum(), -np.median(e)))
    if which == "f":
        assert np.median(best) <= 1e-5 and (best <= 1e-4).sum() >= 56, best
    else:
        assert np.median(best) <= 2e-3, best


def test_tracer_adjoint_configuration_nuh_gradient_zero_for_linear_scheme():
    """With the linear P2 scheme in the tracer-adjoint configuration (depth-uniform flow, ww = 0)
    every layer is advected by the same linear map, so J (the box content summed over the layers)
    is the advection of the column sums, which the vertical diffusion conserves: dJ/dnuh = 0. The
    adjoint's nubar is zero to rounding (relative to the same configuration's dJ/df0)."""
    import torch

    c = cases.streamfunction_flow(nx=256, ny=256, kmax=30, dt=300.0, seed=4)
    c.par.update(cnpar=1.0, avmol=0.0, hscheme=3, vscheme=3)
    ctx, m = make_ctx(c)
    t = _dev_fields(c)
    w = cases.box_weights(c, box=32)
    _, fbar, nubar, _ = _gradient(ctx, c, t, 50, 10, w)
    scale = float(torch.abs(fbar).max()) * float(t["nuh"].max())
    assert float(torch.abs(nubar * t["nuh"]).max()) <= 1e-9 * scale


@pytest.mark.parametrize("which,eps", [("f", 1e-3), ("nuh", 1e-4)])
def test_tracer_adjoint_sheared_linear_scheme_fd(which, eps):
    """The tracer-adjoint configuration with the linear P2 scheme (no branches) and a vertically
    sheared flow (the layers move at 0.5 .. 1.5 times the mean flow, so the vertical diffusion
    changes J): both gradients against central differences on 64 seeded directions, each within
    1e-4 (the step is linear in the tracer, so a large step size only reduces the rounding)."""
    c = cases.streamfunction_flow(nx=256, ny=256, kmax=30, dt=300.0, seed=4, shear=1.0)
    c.par.update(cnpar=1.0, avmol=0.0, hscheme=3, vscheme=3)
    res = _fd_sweep(c, 50, 10, 32, which, (eps,))
    _report(which, res)
    e, _ = res[eps]
    assert e.max() <= 1e-4, e


@pytest.mark.parametrize("scheme,tol", [(3, 1e-4), (4, 1e-3)])
def test_gradient_fp32_vs_fp64_tangent(scheme, tol):
    """FP32 checkpointed gradient against the FP64 tangent-linear oracle. With the linear P2 scheme
    only FP32 rounding separates them (1e-4). With SUPERBEE the FP32 trajectory takes the other
    limiter branch at faces whose limiter ratio sits at a kink within FP32 rounding, so the FP32
    gradient is that of a slightly different piecewise-linear map (1e-3)."""
    import torch

    c = cases.streamfunction_flow(nx=48, ny=40, kmax=8, dt=300.0, seed=4, vertical=0.5, shear=1.0)
    c.par.update(cnpar=0.9, avmol=1e-6, hscheme=scheme, vscheme=scheme)
    p = c.par
    o = oracle.Oracle(c.grid)
    ctx, m = make_ctx(c)
    t32 = _dev_fields(c, torch.float32)
    w = cases.box_weights(c, box=16)
    nsteps, every = 12, 5
    _, fbar, nubar, _ = _gradient(ctx, c, t32, nsteps, every, w, dtype=torch.float32)
    G, NB = host(fbar).astype(np.float64), host(nubar).astype(np.float64)
    rng = np.random.default_rng(6)
    for q in range(4):
        df = rng.normal(size=c["f"].shape) * (c["az"] >= 1)[None]
        dnuh = (rng.normal(size=c["f"].shape) * c["nuh"]) if q % 2 else None
        if dnuh is not None:
            df = np.zeros_like(df)
        fo, dfo = c["f"].copy(), df.copy()
        o.tracer_steps_tl(c.masks(), nsteps, p["dt"], fo, dfo, *[c[n] for n in NAMES], c["nuh"], dnuh, 2,
                          p["hscheme"], p["vscheme"], p["AH"], p["cnpar"], p["avmol"])
        tl = float(np.sum(w * dfo))
        ad = float(np.sum(G * df) + (np.sum(NB * dnuh) if dnuh is not None else 0.0))
        assert abs(ad - tl) <= tol * abs(tl), (q, ad, tl)


def test_adjoint_rejects_other_splits():
    from code_b200.getm import GetmError
    import torch

    c = cases.random_case(nx=20, ny=16, kmax=5, seed=1)
    ctx, m = make_ctx(c)
    t = _dev_fields(c)
    f = dev(c["f"])
    with pytest.raises(GetmError):
        ctx.tracer_step_record(30.0, f, *[t[n] for n in NAMES], t["nuh"], 1, 4, 4, 0.0, 0.9, 0.0,
                               ctx.tape(torch.float64))


@pytest.mark.parametrize("scheme", list(SCHEMES))
@pytest.mark.parametrize("AH", [0.0, 5.0])
def test_fp32_adjoint_vector_and_tile_sweeps_agree(scheme, AH):
    """The vectorised FP32 adjoint sweeps (16-byte aligned rows) agree with the tile sweeps to FP32
    rounding: the cotangents differ by at most 1e-5 of their largest magnitude."""
    import torch

    hs = SCHEMES[scheme]
    c = cases.random_case(nx=60, ny=45, kmax=7, seed=11)
    p = c.par
    p.update(AH=AH, cnpar=0.9, avmol=1e-6)
    ctx, m = make_ctx(c)
    t = _dev_fields(c, torch.float32)
    w = np.random.default_rng(5).normal(size=c["f"].shape)
    out = {}
    prev = G.set_vector_sweeps(True)
    try:
        for on in (True, False):
            G.set_vector_sweeps(on)
            f = dev(c["f"]).to(torch.float32)
            tape = ctx.tape(torch.float32)
            ctx.tracer_step_record(p["dt"], f, *[t[n] for n in NAMES], t["nuh"], 2, hs, hs, AH, p["cnpar"],
                                   p["avmol"], tape)
            fbar = dev(w).to(torch.float32)
            nubar = torch.zeros_like(fbar)
            ctx.tracer_step_adjoint(p["dt"], fbar, nubar, *[t[n] for n in NAMES], t["nuh"], 2, hs, hs, AH,
                                    p["cnpar"], p["avmol"], tape)
            out[on] = (host(fbar).astype(np.float64), host(nubar).astype(np.float64))
    finally:
        G.set_vector_sweeps(prev)
    for a, b in zip(out[True], out[False]):
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()
