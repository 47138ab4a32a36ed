"""The slab decomposition of the tracer step (code_b200/slabs.py) on CPU: world_size 2 and 3 gloo
ranks, each running its slab of rows with the oracle's split sweeps and diffusion solve (the
checker, in place of the library's kernels) and the decomposition's halo-row exchange (packed rows
as torch.distributed point-to-point messages), against the oracle on the undivided domain: every
interior cell bit for bit after several steps (advection_3d.F90's exchange points are enough for
an exact result). The global content from the ranks' compensated partial sums agrees with the
undivided domain's to 1e-15."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

STEPS = 4
SCHEMES = (6, 4)  # P2_PDM, SUPERBEE (horizontal / vertical)
CNPAR, AVMOL, AH = float(np.float32(0.9)), 1.1e-9, -1.0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleSlabPart:
    """One slab's tracer step with the oracle's routines on numpy arrays (test infrastructure: the
    GPU path uses code_b200.slabs.GpuSlabPart, i.e. the library)."""

    def __init__(self, slab, case):
        import oracle

        self.slab = slab
        g = slab.grid
        self.o = oracle.Oracle(g)
        self.t = {k: np.ascontiguousarray(slab.take(case[k])) for k in
                  ("f", "uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")}
        self.t["hu"], self.t["hv"] = self.t["hun"], self.t["hvn"]
        m = [np.ascontiguousarray(slab.take(case[k])) for k in ("az", "au", "av", "ax")]
        self.az = m[0]
        pl = self.o.build_masks(*m)
        self.mflux_u, self.mflux_v, self.mupd = (np.ascontiguousarray(pl[k]) for k in ("uflux", "vflux", "updateH"))
        self.hi = np.empty_like(self.t["f"])
        self.adv = np.zeros_like(self.t["f"])

    def begin(self):
        self.hi[...] = self.t["ho"]
        self.adv[...] = 0.0

    def sweep_u(self, dt, splitfac, scheme, AH):
        t = self.t
        for k in range(1, self.slab.grid.kmax + 1):
            self.o.adv_split_u(dt, t["f"][k], t["f"][k], self.hi[k], self.adv[k], t["uu"][k], t["hu"][k], splitfac,
                               scheme, AH, self.mflux_u, self.mupd)

    def sweep_v(self, dt, splitfac, scheme, AH):
        t = self.t
        for k in range(1, self.slab.grid.kmax + 1):
            self.o.adv_split_v(dt, t["f"][k], t["f"][k], self.hi[k], self.adv[k], t["vv"][k], t["hv"][k], splitfac,
                               scheme, AH, self.mflux_v, self.mupd)

    def sweep_w(self, dt, scheme, tag):
        if self.slab.grid.kmax > 1:
            t = self.t
            self.o.adv_split_w(dt, t["f"], t["f"], self.hi, self.adv, t["ww"], 1.0, scheme, tag, self.az, 1)

    def vdiff(self, dt, cnpar, avmol):
        t = self.t
        self.o.tracer_vdiff(dt, cnpar, avmol, t["f"], t["hn"], t["nuh"], self.az)

    def pack(self, name, j_first):
        import torch

        r = j_first - (1 - 2)  # array row of reference row j_first (local jmin = 1)
        return torch.from_numpy(np.ascontiguousarray(self.t[name][:, r:r + 2, :]))

    def unpack(self, name, j_first, buf):
        r = j_first - (1 - 2)
        self.t[name][:, r:r + 2, :] = buf.numpy()


def _case():
    from code_b200 import cases

    return cases.random_case(nx=23, ny=21, kmax=6, seed=12, land=0.25, open_bdy=True)


def _single_domain(c):
    import oracle

    o = oracle.Oracle(c.grid)
    f = c["f"].copy()
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    o.tracer_steps(c.masks(), STEPS, c.par["dt"], f, *[c[n] for n in names], 2, SCHEMES[0], SCHEMES[1], AH, CNPAR,
                   AVMOL)
    return f


def _rank(rank, world, port, out):
    import torch.distributed as dist

    from code_b200 import slabs
    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = _case()
        sl = slabs.slabs_of(c.grid, world)[rank]
        part = OracleSlabPart(sl, c)
        ex = slabs.RowExchange({rank: part}, dist)
        for _ in range(STEPS):
            slabs.tracer_step({rank: part}, ex, c.par["dt"], SCHEMES[0], SCHEMES[1], AH, CNPAR, AVMOL)
        # compensated partial content of the slab's cells (Neumaier over k, j, i) and its error term
        g = sl.grid
        s = comp = 0.0
        f, h, az = part.t["f"], part.t["hn"], part.az
        for k in range(1, g.kmax + 1):
            for j in range(2, 2 + g.ny):
                for i in range(2, 2 + g.nx):
                    if az[j, i] < 1:
                        continue
                    x = float(f[k, j, i]) * float(h[k, j, i]) / g.ard1
                    t = s + x
                    comp += (s - t) + x if abs(s) >= abs(x) else (x - t) + s
                    s = t
        total = slabs.global_content((s, comp), dist)
        out[rank] = (sl.j0, sl.ny, part.t["f"][:, sl.interior(), :].copy(), total)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_slabs_in_one_process_match_single_domain(world):
    """All slabs held by one process (their exchange is a copy between the parts, the form the GPU
    test on one device uses), slabs of unequal row counts (21 rows into 11 + 10, 7 + 7 + 7 and
    6 + 5 + 5 + 5): every interior cell bit for bit after several steps."""
    from code_b200 import slabs

    c = _case()
    want = _single_domain(c)
    parts = {sl.rank: OracleSlabPart(sl, c) for sl in slabs.slabs_of(c.grid, world)}
    ex = slabs.RowExchange(parts)
    for _ in range(STEPS):
        slabs.tracer_step(parts, ex, c.par["dt"], SCHEMES[0], SCHEMES[1], AH, CNPAR, AVMOL)
    got = want.copy()
    got[:, 2:-2, :] = np.nan
    for p in parts.values():
        p.slab.put(p.t["f"], got)
    assert np.array_equal(got[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2])


@pytest.mark.parametrize("world", [2, 3])
def test_slab_tracer_steps_match_single_domain(world):
    import oracle

    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        res = dict(out)
    c = _case()
    want = _single_domain(c)
    got = want.copy()
    got[:, 2:-2, :] = np.nan
    for r in range(world):
        j0, ny, fint, _ = res[r]
        got[:, 2 + j0 - 1:2 + j0 - 1 + ny, :] = fint
    assert np.array_equal(got[:, 2:-2, :], want[:, 2:-2, :])
    o = oracle.Oracle(c.grid)
    total = o.tracer_content(want, c["hn"], c["az"])
    for r in range(world):
        assert res[r][3] == res[0][3]  # every rank gets the same sum
        assert abs(res[r][3] - total) <= 1e-15 * abs(total)


def test_row_split():
    from code_b200.slabs import row_split

    assert row_split(21, 3) == [(1, 7), (8, 7), (15, 7)]
    assert row_split(10, 3) == [(1, 4), (5, 3), (8, 3)]
    with pytest.raises(ValueError):
        row_split(5, 3)
