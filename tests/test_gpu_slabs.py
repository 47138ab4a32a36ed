"""The slab decomposition of the tracer step on the GPU: two and three slabs of one domain held by
one process (their halo-row exchange is the library's pack / unpack kernels with a device copy in
between -- no kernels that wait on one another), each stepped by the library's sweeps and diffusion
solve, against the undivided domain's getm_tracer_step: every interior cell bit for bit, FP64 and
FP32. And the GPU slabs against the oracle's slabs (the checker of the decomposition on CPU) after
every phase of two steps: whole slabs, halo rows and columns included, FP64 bit for bit. The halo pack / unpack kernels are also checked against plain row slicing."""
import numpy as np
import pytest

from code_b200 import cases, slabs
from code_b200.getm import Context
from helpers import dev, host

pytestmark = pytest.mark.gpu

NAMES = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["fp64", "fp32"])
def test_slabs_match_single_domain(world, dtype):
    import torch

    c = cases.random_case(nx=37, ny=31, kmax=7, seed=12, land=0.25, open_bdy=True, dtype=dtype)
    p = dict(dt=c.par["dt"], hs=6, vs=4, AH=-1.0, cnpar=float(np.float32(0.9)), avmol=1.1e-9)
    # the undivided domain
    ctx = Context(c.grid)
    ctx.init_advection(*[dev(m) for m in c.masks()])
    f = dev(c["f"])
    t = [dev(c[n]) for n in NAMES]
    for _ in range(4):
        ctx.tracer_step(p["dt"], f, *t, 2, p["hs"], p["vs"], p["AH"], p["cnpar"], p["avmol"])
    want = host(f)
    # the slabs
    parts = {}
    for sl in slabs.slabs_of(c.grid, world):
        cx = Context(sl.grid)
        m = [dev(sl.take(a)) for a in c.masks()]
        cx.init_advection(*m)
        tt = {n: dev(sl.take(c[n])) for n in ("f",) + NAMES}
        parts[sl.rank] = slabs.GpuSlabPart(sl, cx, tt["f"], tt["uu"], tt["vv"], tt["ww"], tt["hun"], tt["hvn"],
                                           tt["ho"], tt["hn"], tt["nuh"], m[0])
    ex = slabs.RowExchange(parts)
    for _ in range(4):
        slabs.tracer_step(parts, ex, p["dt"], p["hs"], p["vs"], p["AH"], p["cnpar"], p["avmol"])
    torch.cuda.synchronize()
    got = want.copy()
    got[:, 2:-2, :] = np.nan
    for r, part in parts.items():
        part.slab.put(host(part.t["f"]), got)
    # the interior cells (the halo columns of a closed domain are land, where the undivided step's
    # scratch ping-pong and the slabs' in-place sweeps leave different bytes)
    assert np.array_equal(got[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2])


def test_halo_pack_unpack_rows():
    import torch

    c = cases.random_case(nx=13, ny=11, kmax=5, seed=3)
    ctx = Context(c.grid)
    for dtype in (torch.float64, torch.float32):
        f = dev(c["f"]).to(dtype)
        buf = torch.empty((6, 2, c.grid.ni), dtype=dtype, device="cuda")
        ctx.halo_pack(f, 4, 2, buf)  # rows j = 4, 5: array rows 5, 6
        torch.cuda.synchronize()
        assert torch.equal(buf, f[:, 5:7, :])
        g = torch.zeros_like(f)
        ctx.halo_unpack(g, 0, 2, buf)  # into rows j = 0, 1: array rows 1, 2
        torch.cuda.synchronize()
        assert torch.equal(g[:, 1:3, :], f[:, 5:7, :])
        assert float(g[:, 3:, :].abs().max()) == 0.0 and float(g[:, 0, :].abs().max()) == 0.0


def test_slab_phases_vs_oracle_slabs():
    import torch

    from test_slabs_cpu import OracleSlabPart

    c = cases.random_case(nx=37, ny=31, kmax=7, seed=12, land=0.25, open_bdy=True)
    dt, hs, vs, AH, cnpar, avmol = c.par["dt"], 6, 4, -1.0, float(np.float32(0.9)), 1.1e-9
    gp, op = {}, {}
    for sl in slabs.slabs_of(c.grid, 2):
        cx = Context(sl.grid)
        m = [dev(sl.take(a)) for a in c.masks()]
        cx.init_advection(*m)
        tt = {n: dev(sl.take(c[n])) for n in ("f",) + NAMES}
        gp[sl.rank] = slabs.GpuSlabPart(sl, cx, tt["f"], tt["uu"], tt["vv"], tt["ww"], tt["hun"], tt["hvn"],
                                        tt["ho"], tt["hn"], tt["nuh"], m[0])
        op[sl.rank] = OracleSlabPart(sl, c)
    gx, ox = slabs.RowExchange(gp), slabs.RowExchange(op)
    phases = [lambda p: p.begin(), lambda p: p.sweep_u(dt, 0.5, hs, AH), lambda p: p.sweep_v(dt, 0.5, hs, AH),
              lambda p: p.sweep_w(dt, vs, 10), None, lambda p: p.sweep_v(dt, 0.5, hs, AH),
              lambda p: p.sweep_u(dt, 0.5, hs, AH), lambda p: p.vdiff(dt, cnpar, avmol), None]
    for step in range(2):
        for q, fn in enumerate(phases):
            if fn is None:
                gx.exchange("f")
                ox.exchange("f")
            else:
                for r in gp:
                    fn(gp[r])
                    fn(op[r])
            torch.cuda.synchronize()
            for r in gp:
                assert np.array_equal(host(gp[r].t["f"]), op[r].t["f"]), (step, q, r)
                assert np.array_equal(host(gp[r].hi), op[r].hi), (step, q, r)
