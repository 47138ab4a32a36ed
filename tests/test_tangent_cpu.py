"""The oracle's tangent-linear tracer step (dual numbers, oracle/getm_tangent.hpp) -- the FP64
reference gradient the GPU adjoint is checked against. Here it is checked on the CPU: its values
equal the plain FP64 oracle bit for bit, and its directional derivatives agree with central
finite differences of the plain oracle."""
import numpy as np
import pytest

import oracle
from code_b200 import cases

NAMES = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn")


def _run(o, c, f, nuh, nsteps):
    p = c.par
    f = f.copy()
    o.tracer_steps(c.masks(), nsteps, p["dt"], f, *[c[n] for n in NAMES], nuh, p["split"], p["hscheme"],
                   p["vscheme"], p["AH"], p["cnpar"], p["avmol"])
    return f


def _tl(o, c, f, df, nuh, dnuh, nsteps):
    p = c.par
    f, df = f.copy(), df.copy()
    o.tracer_steps_tl(c.masks(), nsteps, p["dt"], f, df, *[c[n] for n in NAMES], nuh, dnuh, p["split"],
                      p["hscheme"], p["vscheme"], p["AH"], p["cnpar"], p["avmol"])
    return f, df


@pytest.fixture(scope="module")
def flow():
    c = cases.streamfunction_flow(nx=24, ny=20, kmax=6, dt=300.0, seed=4)
    c.par.update(cnpar=0.9, avmol=1e-6)
    return c


def test_tangent_values_equal_plain_oracle(flow):
    o = oracle.Oracle(flow.grid)
    rng = np.random.default_rng(1)
    df = rng.normal(size=flow["f"].shape)
    plain = _run(o, flow, flow["f"], flow["nuh"], 5)
    val, _ = _tl(o, flow, flow["f"], df, flow["nuh"], None, 5)
    assert np.array_equal(val, plain)


@pytest.mark.parametrize("which", ["f", "nuh"])
def test_tangent_matches_central_differences(flow, which):
    o = oracle.Oracle(flow.grid)
    rng = np.random.default_rng(2 if which == "f" else 3)
    w = rng.normal(size=flow["f"].shape)
    nsteps = 5
    f0, nuh = flow["f"], flow["nuh"]
    d = rng.normal(size=f0.shape) * (1e-3 if which == "f" else 1e-5)
    zero = np.zeros_like(f0)
    if which == "f":
        _, df = _tl(o, flow, f0, d, nuh, None, nsteps)
        # small enough that no limiter branch flips between f0 - eps*d and f0 + eps*d
        eps = 1e-5
        jp = np.sum(w * _run(o, flow, f0 + eps * d, nuh, nsteps))
        jm = np.sum(w * _run(o, flow, f0 - eps * d, nuh, nsteps))
    else:
        _, df = _tl(o, flow, f0, zero, nuh, d, nsteps)
        eps = 1e-3
        jp = np.sum(w * _run(o, flow, f0, nuh + eps * d, nsteps))
        jm = np.sum(w * _run(o, flow, f0, nuh - eps * d, nsteps))
    tl = np.sum(w * df)
    fd = (jp - jm) / (2 * eps)
    assert abs(tl - fd) <= 1e-6 * max(abs(tl), 1e-30), (tl, fd)
