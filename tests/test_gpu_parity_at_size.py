"""FP64 parity of the mode-split step at the configurations' sizes, cell by cell.

The GPU step (getm_time_loop, plain FP64) and the oracle run the same seeded inputs:
  * the tidal-shelf configuration: 512 x 512 x 30 sigma layers, shelf bathymetry, dx = 1 km, M = 20
    (dt = 60 s), M2 tide of 1 m amplitude (period 44714.16 s) clamped on the western boundary,
    P2_PDM / HALFSPLIT, Blumberg-Mellor, prescribed parabolic viscosity; 3 macro steps;
  * a 256 x 256 x 50 sample of the large irregular domain (30% land from Gaussian-smoothed noise,
    islands kept, depth 5-150 m), closed; 3 macro steps.

Metric, per cell of every 2D and 3D field: |gpu - oracle| <= 1e-12 * max(|oracle|, floor), with
floor = 1e-3 * max|oracle field|: the relative error of each cell, measured against its own value
where that value is at least a thousandth of the field's scale, and against that thousandth where a
field crosses zero. Such cells (velocities, transports, the vertical velocity of the continuity
integral, gradients) are sums of terms of the field's scale and carry their absolute rounding, which
relative to a value near zero is unbounded. All arithmetic is the reference's, in its order, without
contraction; the one difference is the device's natural logarithm in the log-law drag
(bottom_friction.F90, bottom_friction_3d.F90, slow_bottom_friction.F90), which may differ from the
host C library's in the last bit. The test prints, per field, the share of bit-identical cells and
the largest per-cell error with floors of 1e-6, 1e-4 and 1e-3 of the scale (pytest -s). Also
checked: the tracer content of the closed sample (compensated sum) agrees with the oracle's to
1e-13.
"""
import numpy as np
import pytest

import oracle
from code_b200 import state as S
from code_b200.getm import BcDevice
from helpers import make_ctx

pytestmark = pytest.mark.gpu

REL = 1e-12
FLOOR = 1e-3
FLOORS = (1e-6, 1e-4, 1e-3)


def cellwise(a, b, floor=FLOOR):
    """Largest per-cell error |a-b| / max(|b|, floor*max|b|) of one field (0 for an all-zero field)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = float(np.nanmax(np.abs(b))) if b.size else 0.0
    if scale == 0.0:
        return float(np.nanmax(np.abs(a))) if a.size else 0.0
    den = np.maximum(np.abs(b), floor * scale)
    return float(np.nanmax(np.abs(a - b) / den))


def run_both(c, n_micro):
    import torch

    ref = c.copy()
    oracle.bc_steps(ref, 1, n_micro)
    ctx, _ = make_ctx(c)
    if c.bdy is not None:
        ctx.set_open_boundaries(c.bdy)
    st = BcDevice(c)
    ctx.time_loop(st, 1, n_micro)
    torch.cuda.synchronize()
    out = st.to_host(c.copy())
    return out, ref, ctx, st


def check_cellwise(out, ref, label):
    worst = {}
    lines = [f"{label}: field, bit-identical share, max per-cell error at floors {FLOORS}"]
    pairs = [("f2_" + k, out.f2[k], ref.f2[k]) for k in S.F2_NAMES] + \
            [("f3_" + k, out.f3[k], ref.f3[k]) for k in S.F3_NAMES]
    for name, a, b in pairs:
        worst[name] = cellwise(a, b)
        same = float(np.mean((np.asarray(a, np.float64) == np.asarray(b, np.float64)) | (np.isnan(a) & np.isnan(b))))
        lines.append(f"  {name:10s} {same:.6f} " + " ".join(f"{cellwise(a, b, fl):.2e}" for fl in FLOORS))
    print("\n".join(lines))
    bad = {k: v for k, v in worst.items() if not v <= REL}
    return bad, worst


def test_tidal_shelf_512x512x30_cellwise():
    g = S.Grid(512, 512, 30, 1000.0, 1000.0)
    b = S.OpenBoundaries(west=[(g.imin, g.jmin, g.jmax, S.CLAMPED)], amp=1.0, period=44714.16)
    c = S.baroclinic_case(nx=512, ny=512, kmax=30, recipe="shelf", M=20, dt3=60.0, seed=3, bdy=b)
    out, ref, _, _ = run_both(c, 3 * 20)
    bad, worst = check_cellwise(out, ref, "tidal shelf 512x512x30")
    assert not bad, bad
    # the tide entered: boundary elevations follow the M2 forcing
    assert np.abs(out.f2["z"][:, 2]).max() > 1e-3


def test_islands_sample_256x256x50_cellwise_and_content():
    c = S.baroclinic_case(nx=256, ny=256, kmax=50, recipe="islands", land=0.3, M=20, dt3=60.0, seed=6)
    out, ref, ctx, st = run_both(c, 3 * 20)
    bad, worst = check_cellwise(out, ref, "islands 256x256x50")
    assert not bad, bad
    o = oracle.Oracle(c.grid)
    for name in ("T", "S"):
        want = o.tracer_content(ref.f3[name], ref.f3["hn"], c.az)
        got = ctx.tracer_content(st.t["f3_" + name], st.t["f3_hn"], st.t["az"])
        assert abs(got - want) <= 1e-13 * abs(want), (name, got, want)
