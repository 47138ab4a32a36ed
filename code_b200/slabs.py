"""A GETM domain cut into slabs of rows (a 1D decomposition in j) over ranks, with the halo
exchange of the reference's parallel build, for the tracer step (do_advection_3d with HALFSPLIT
and the implicit vertical diffusion of do_salinity / do_temperature).

Reference: the MPI decomposition of halo_mpi.F90:376-558 exchanges the HALO = 2 rows (and
columns) next to each subdomain boundary. The tracer step exchanges the tracer where the next sweep
reads rows that its own sweeps cannot update (advection_3d.F90:456-527, HALFSPLIT: before the
second v/2 sweep -- for UPSTREAM only on the V grid -- and before the second u/2 sweep, which a
decomposition in j alone does not need), and integrate_3d exchanges the new tracer after the
diffusion (m3d.F90:583-593). Every other input
(transports, layer heights, masks) is given with valid halo rows, so each rank computes the layer
heights of its halo rows itself (the reference never exchanges them).

A slab holds the interior rows j0 .. j0+ny-1 of the global domain (reference indices, 1-based)
plus two halo rows on each side, laid out exactly like a whole domain of ny rows; its local grid
numbers the rows 1 .. ny. Neighbours are the slabs of the rows above (north, rank + 1) and below
(south, rank - 1); the outermost slabs keep the global halo rows (closed boundaries: land).

The exchange moves, per neighbour, two packed rows of every level: the library's pack / unpack
kernels (getm_halo_pack / getm_halo_unpack) and, between processes, torch.distributed point-to-
point messages (NCCL between GPUs); between two slabs of one process a device copy. No
collective other than the compensated content sum (:func:`global_content`) is used.
"""
from __future__ import annotations

from dataclasses import dataclass

from .grid import HALO, Grid

H_TAG, U_TAG, V_TAG = 10, 31, 32
UPSTREAM = 1


def row_split(ny: int, world: int) -> list[tuple[int, int]]:
    """(first global interior row, number of rows) of each rank: near-equal contiguous slabs, the
    first ny % world ranks one row larger. Every slab needs at least HALO rows."""
    if world < 1 or ny < world * HALO:
        raise ValueError(f"cannot cut {ny} rows into {world} slabs of at least {HALO} rows")
    base, extra = divmod(ny, world)
    out, j0 = [], 1
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((j0, n))
        j0 += n
    return out


@dataclass
class Slab:
    """One rank's rows of a global grid."""

    rank: int
    world: int
    j0: int          # first global interior row (reference index, the global grid's jmin = 1)
    ny: int          # interior rows
    glob: Grid       # the whole domain

    @property
    def grid(self) -> Grid:
        g = self.glob
        return Grid(g.nx, self.ny, g.kmax, g.dx, g.dy)

    @property
    def north(self):
        return self.rank + 1 if self.rank + 1 < self.world else None

    @property
    def south(self):
        return self.rank - 1 if self.rank > 0 else None

    def rows(self) -> slice:
        """Array rows (axis -2) of the global haloed field that this slab holds, halos included."""
        a0 = self.j0 - 1  # global array row of local array row 0 (global row j0 - HALO)
        return slice(a0, a0 + self.ny + 2 * HALO)

    def take(self, a):
        """The slab's part of a global field (numpy or torch; 2D or 3D), halo rows included, as a
        new contiguous array."""
        part = a[..., self.rows(), :]
        return part.copy() if hasattr(part, "copy") and not hasattr(part, "clone") else part.clone()

    def interior(self) -> slice:
        """Local array rows of the interior."""
        return slice(HALO, HALO + self.ny)

    def put(self, a_local, a_global):
        """Write the slab's interior rows into the global field."""
        g0 = self.j0 - 1 + HALO
        a_global[..., g0:g0 + self.ny, :] = a_local[..., self.interior(), :]


def slabs_of(glob: Grid, world: int) -> list[Slab]:
    return [Slab(r, world, j0, n, glob) for r, (j0, n) in enumerate(row_split(glob.ny, world))]


class RowExchange:
    """The halo-row exchange of the slabs that one process holds.

    parts: {rank: SlabPart} of this process (one part per process across ranks, or several parts
    in one process -- then their exchange is a device copy). Remote neighbours are reached with
    torch.distributed point-to-point messages of packed rows (the process group's backend: NCCL
    for CUDA tensors, gloo for CPU tensors)."""

    def __init__(self, parts: dict, dist=None):
        self.parts = parts
        self.dist = dist

    def exchange(self, name: str):
        """Bring the two halo rows of field `name` on both sides of every held slab up to date."""
        import torch

        sends, recvs, ops = [], [], []
        for r, p in self.parts.items():
            s = p.slab
            for nb, first in ((s.north, s.ny - HALO + 1), (s.south, 1)):
                # rows first..first+1 of this slab go into the neighbour's halo rows on this side:
                # rows 1-HALO.. of the northern neighbour, rows ny+1.. (its own ny) of the southern one
                if nb is None:
                    continue
                buf = p.pack(name, first)
                if nb in self.parts:
                    dst_first = 1 - HALO if nb == s.north else self.parts[nb].slab.ny + 1
                    self.parts[nb].unpack(name, dst_first, buf)
                else:
                    sends.append(buf)
                    ops.append(self.dist.P2POp(self.dist.isend, buf, nb))
                    rb = torch.empty_like(buf)
                    # what the neighbour sends lands in this slab's halo on that side
                    recvs.append((p, name, 1 - HALO if nb == s.south else s.ny + 1, rb))
                    ops.append(self.dist.P2POp(self.dist.irecv, rb, nb))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
            for p, nm, first, rb in recvs:
                p.unpack(nm, first, rb)


def tracer_step(parts: dict, ex: RowExchange, dt: float, hscheme: int, vscheme: int, AH: float, cnpar: float,
                avmol: float, tag: int = H_TAG):
    """One tracer step (do_advection_3d with HALFSPLIT, then the implicit vertical diffusion) on
    every held slab, with the reference's halo exchanges; the tracer's halo rows are up to date on
    entry and on exit."""
    ps = list(parts.values())
    for p in ps:
        p.begin()
    for p in ps:
        p.sweep_u(dt, 0.5, hscheme, AH)
    if hscheme != UPSTREAM and tag == V_TAG:
        ex.exchange("f")
    for p in ps:
        p.sweep_v(dt, 0.5, hscheme, AH)
    for p in ps:
        p.sweep_w(dt, vscheme, tag)
    if hscheme != UPSTREAM or tag == V_TAG:  # advection_3d.F90:478-495
        ex.exchange("f")
    for p in ps:
        p.sweep_v(dt, 0.5, hscheme, AH)
    # advection_3d.F90:506-523 exchanges here as well, for the halo COLUMNS that the second u/2
    # sweep reads in a decomposition in i; a slab's u/2 sweep reads only its own rows, and its
    # halo rows are refreshed after the diffusion
    for p in ps:
        p.sweep_u(dt, 0.5, hscheme, AH)
    for p in ps:
        p.vdiff(dt, cnpar, avmol)
    ex.exchange("f")  # m3d.F90:583-593: the new tracer's halo rows


class GpuSlabPart:
    """One slab's tracer step on the GPU through the library (a Context of the slab's grid)."""

    def __init__(self, slab: Slab, ctx, f, uu, vv, ww, hu, hv, ho, hn, nuh, az, adv_iters=1):
        import torch

        self.slab, self.ctx = slab, ctx
        self.t = dict(f=f, uu=uu, vv=vv, ww=ww, hu=hu, hv=hv, ho=ho, hn=hn, nuh=nuh)
        self.az = az
        self.hi = torch.empty_like(f)
        self.adv = torch.zeros_like(f)
        self.iters = adv_iters
        self.gh = ctx.adv_grid(H_TAG)
        g = slab.grid
        self._buf = torch.empty((g.kmax + 1, HALO, g.ni), dtype=f.dtype, device=f.device)

    def begin(self):
        self.hi.copy_(self.t["ho"])
        self.adv.zero_()

    def sweep_u(self, dt, splitfac, scheme, AH):
        t, k = self.t, self.slab.grid.kmax
        self.ctx.adv_split_u(dt, t["f"][1:], t["f"][1:], self.hi[1:], self.adv[1:], t["uu"][1:], t["hu"][1:],
                             splitfac, scheme, AH, self.gh.mask_uflux, self.gh.mask_uupdate, nk=k)

    def sweep_v(self, dt, splitfac, scheme, AH):
        t, k = self.t, self.slab.grid.kmax
        self.ctx.adv_split_v(dt, t["f"][1:], t["f"][1:], self.hi[1:], self.adv[1:], t["vv"][1:], t["hv"][1:],
                             splitfac, scheme, AH, self.gh.mask_vflux, self.gh.mask_vupdate, nk=k)

    def sweep_w(self, dt, scheme, tag):
        if self.slab.grid.kmax > 1:
            t = self.t
            self.ctx.adv_split_w(dt, t["f"], t["f"], self.hi, self.adv, t["ww"], 1.0, scheme, tag, self.az,
                                 self.iters)

    def vdiff(self, dt, cnpar, avmol):
        t = self.t
        self.ctx.tracer_vdiff(dt, cnpar, avmol, t["f"], t["hn"], t["nuh"], self.az)

    def pack(self, name, j_first):
        buf = self._buf.clone()
        self.ctx.halo_pack(self.t[name], j_first, HALO, buf)
        return buf

    def unpack(self, name, j_first, buf):
        self.ctx.halo_unpack(self.t[name], j_first, HALO, buf)


def global_content(partial: tuple[float, float], dist=None) -> float:
    """The global tracer content from each rank's compensated partial sum (s, c) -- the Neumaier sum
    and its carried error of the rank's cells: the pairs of all ranks are gathered and combined on
    every rank in rank order with the same compensated summation, so every rank gets the same
    value, and it does not depend on message timing."""
    import torch

    pair = torch.tensor(partial, dtype=torch.float64)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        pairs = [pair]
    else:
        if dist.get_backend() == "nccl":
            pair = pair.cuda()
        pairs = [torch.zeros_like(pair) for _ in range(dist.get_world_size())]
        dist.all_gather(pairs, pair)
    s = comp = 0.0
    for p in pairs:
        for x in (float(p[0]), float(p[1])):
            t = s + x
            comp += (s - t) + x if abs(s) >= abs(x) else (x - t) + s
            s = t
    return s + comp
