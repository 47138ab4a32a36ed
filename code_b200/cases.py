"""Seeded synthetic inputs for the hot path (no datasets are involved).

* :func:`tracer_rotation` -- solid-body rotation of a Gaussian tracer blob in a closed flat
  basin (the 128x128x20 plain-FP64 tracer advection-diffusion case and its scaled versions).
* :func:`random_case` -- random fields over a random land mask, for cell-wise parity tests of the
  individual routines (limiter branches, masks, open-boundary mask values 2/3 all exercised).

All arrays are numpy, C-contiguous, in the reference layout (:mod:`code_b200.grid`).
"""
from __future__ import annotations

import numpy as np

from .grid import HALO, Grid


def derive_uvx(az: np.ndarray):
    """au, av, ax from az over the haloed range (domain.F90:292-346)."""
    a, b = az[:, :-1], az[:, 1:]
    au = np.zeros_like(az)
    u = np.zeros_like(a)
    u[(a == 1) & (b == 1)] = 1
    u[((a == 1) & (b == 2)) | ((a == 2) & (b == 1))] = 2
    u[(a == 2) & (b == 2)] = 3
    au[:, :-1] = u
    a, b = az[:-1, :], az[1:, :]
    av = np.zeros_like(az)
    v = np.zeros_like(a)
    v[(a == 1) & (b == 1)] = 1
    v[((a == 1) & (b == 2)) | ((a == 2) & (b == 1))] = 2
    v[(a == 2) & (b == 2)] = 3
    av[:-1, :] = v
    ax = np.zeros_like(az)
    ax[:-1, :-1] = ((az[:-1, :-1] >= 1) & (az[1:, :-1] >= 1) & (az[:-1, 1:] >= 1) & (az[1:, 1:] >= 1)).astype(az.dtype)
    return au, av, ax


def closed_basin(g: Grid) -> np.ndarray:
    az = np.zeros(g.shape2(), np.int32)
    az[g.interior()] = 1
    return az


class Case(dict):
    """Dict of named arrays plus scalar parameters in ``.par``."""

    def __init__(self, grid: Grid, **kw):
        super().__init__(**kw)
        self.grid = grid
        self.par = {}

    def masks(self):
        return self["az"], self["au"], self["av"], self["ax"]


def tracer_rotation(nx=128, ny=128, kmax=20, depth=20.0, dx=500.0, dt=10.0, umax=1.0, sigma_cells=8.0,
                    noise=1e-3, nuh=1e-4, seed=1, dtype=np.float64) -> Case:
    """Solid-body rotation of a tracer blob in a closed, flat basin.

    Velocity from a discrete streamfunction at X-points, psi = 0.5*omega*min(r,R)^2 with R = nx/2
    cells and omega = umax/R, so the transports are discretely divergence-free and the normal
    flux through the walls is zero; ww = 0. Tracer: Gaussian (amplitude 1, sigma = sigma_cells)
    centred at (0.3 nx, 0.5 ny) plus uniform noise in [-noise, noise] (seeded).
    """
    g = Grid(nx, ny, kmax, dx, dx)
    rng = np.random.default_rng(seed)
    az = closed_basin(g)
    au, av, ax = derive_uvx(az)
    h = depth / kmax
    # reference index vectors over the haloed range
    i = np.arange(g.imin - HALO, g.imax + HALO + 1)
    j = np.arange(g.jmin - HALO, g.jmax + HALO + 1)
    # X-point (i,j) is the north-east corner of T-cell (i,j): x = (i-imin+1)*dx
    xX = (i - g.imin + 1) * dx
    yX = (j - g.jmin + 1) * dx
    xc, yc = nx * dx / 2, ny * dx / 2
    R = (nx / 2) * dx
    om = umax / R
    r = np.sqrt((xX[None, :] - xc) ** 2 + (yX[:, None] - yc) ** 2)
    psi = 0.5 * om * np.minimum(r, R) ** 2
    u = np.zeros(g.shape2())
    v = np.zeros(g.shape2())
    u[1:, :] = -(psi[1:, :] - psi[:-1, :]) / dx  # U(i,j) between X(i,j-1) and X(i,j)
    v[:, 1:] = (psi[:, 1:] - psi[:, :-1]) / dx   # V(i,j) between X(i-1,j) and X(i,j)
    u *= (au == 1)
    v *= (av == 1)
    shp = g.shape3()
    hh = np.full(shp, h)
    hh[0] = 0.0
    uu = np.zeros(shp)
    vv = np.zeros(shp)
    uu[1:] = u[None] * h
    vv[1:] = v[None] * h
    ww = np.zeros(shp)
    xT = (i - g.imin + 0.5) * dx
    yT = (j - g.jmin + 0.5) * dx
    x0, y0 = 0.3 * nx * dx, 0.5 * ny * dx
    s = sigma_cells * dx
    blob = np.exp(-((xT[None, :] - x0) ** 2 + (yT[:, None] - y0) ** 2) / (2 * s * s))
    f = np.zeros(shp)
    f[1:] = blob[None]
    f[1:] += rng.uniform(-noise, noise, size=(kmax, g.nj, g.ni))
    f *= (az >= 1)[None]
    c = Case(g, az=az, au=au, av=av, ax=ax, f=f.astype(dtype), uu=uu.astype(dtype), vv=vv.astype(dtype),
             ww=ww.astype(dtype), ho=hh.astype(dtype), hn=hh.copy().astype(dtype), hun=hh.copy().astype(dtype),
             hvn=hh.copy().astype(dtype), nuh=np.full(shp, nuh, dtype=dtype))
    c.par.update(dt=dt, split=2, hscheme=4, vscheme=4, AH=0.0, cnpar=1.0, avmol=0.0, adv_ver_iterations=1)
    return c


def tracer_rotation_device(nx=2048, ny=2048, kmax=50, depth=50.0, dx=1000.0, dt=60.0, umax=1.0,
                           sigma_cells=64.0, noise=1e-3, nuh=1e-4, seed=1, dtype=None, device="cuda"):
    """The rotation case built directly on the device (for sizes whose 3D fields would not fit
    comfortably in host memory). The 2D parts are computed in numpy exactly as in
    :func:`tracer_rotation`; the 3D noise comes from a seeded device generator. Returns
    (grid, dict of tensors, par)."""
    import torch

    dtype = dtype or torch.float64
    small = tracer_rotation(nx=nx, ny=ny, kmax=1, depth=depth / kmax, dx=dx, dt=dt, umax=umax,
                            sigma_cells=sigma_cells, noise=0.0, nuh=nuh, seed=seed)
    g = Grid(nx, ny, kmax, dx, dx)
    h = depth / kmax
    shp = g.shape3()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    u2 = t(small["uu"][1] / (depth / kmax)).to(dtype)
    v2 = t(small["vv"][1] / (depth / kmax)).to(dtype)
    blob = t(small["f"][1]).to(dtype)
    wet = t((small["az"] >= 1).astype(np.float64)).to(dtype)
    out = {}
    hh = torch.full(shp, h, dtype=dtype, device=device)
    hh[0] = 0
    for n in ("ho", "hn", "hun", "hvn"):
        out[n] = hh.clone()
    uu = torch.zeros(shp, dtype=dtype, device=device)
    vv = torch.zeros(shp, dtype=dtype, device=device)
    uu[1:] = u2 * h
    vv[1:] = v2 * h
    out["uu"], out["vv"] = uu, vv
    out["ww"] = torch.zeros(shp, dtype=dtype, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    f = torch.zeros(shp, dtype=dtype, device=device)
    f[1:] = blob + (torch.rand((kmax,) + g.shape2(), generator=gen, device=device, dtype=torch.float64) * 2 - 1
                    ).to(dtype) * noise
    f *= wet
    out["f"] = f
    out["nuh"] = torch.full(shp, nuh, dtype=dtype, device=device)
    for n in ("az", "au", "av", "ax"):
        out[n] = t(small[n])
    par = dict(small.par)
    return g, out, par


def streamfunction_flow(nx=256, ny=256, kmax=30, depth=30.0, dx=500.0, dt=300.0, umax=0.5, modes=8,
                        sigma_cells=16.0, noise=1e-3, nuh=1e-4, seed=4, vertical=0.0, slope=0.0, shear=0.0,
                        dtype=np.float64) -> Case:
    """Tracer advection-diffusion in a closed flat basin driven by a random divergence-free flow
    (the tracer-adjoint configuration).

    Streamfunction at X-points psi = sum over `modes` seeded (m, n) in 1..8 of
    a_mn sin(m pi x/Lx) sin(n pi y/Ly), a_mn ~ N(0,1), scaled so that max |u|, |v| = umax; the
    transports are its discrete curl (divergence-free, zero normal flux at the walls), ww = 0; with
    shear > 0 layer k carries the flow times 1 + shear*((k-1/2)/kmax - 1/2) (still divergence-free
    in every layer).
    Tracer: a centred Gaussian (sigma = sigma_cells), times 1 + vertical*cos(pi*(k-1/2)/kmax) on
    layer k, plus slope*(x/Lx + y/Ly) and uniform noise. SUPERBEE, HALFSPLIT, implicit diffusion
    with constant nuh.
    """
    g = Grid(nx, ny, kmax, dx, dx)
    rng = np.random.default_rng(seed)
    az = closed_basin(g)
    au, av, ax = derive_uvx(az)
    h = depth / kmax
    i = np.arange(g.imin - HALO, g.imax + HALO + 1)
    j = np.arange(g.jmin - HALO, g.jmax + HALO + 1)
    Lx, Ly = nx * dx, ny * dx
    xX = np.clip((i - g.imin + 1) * dx, 0.0, Lx)
    yX = np.clip((j - g.jmin + 1) * dx, 0.0, Ly)
    psi = np.zeros(g.shape2())
    mn = rng.integers(1, 9, size=(modes, 2))
    amp = rng.normal(size=modes)
    for (m, n), a in zip(mn, amp):
        psi += a * np.sin(m * np.pi * xX[None, :] / Lx) * np.sin(n * np.pi * yX[:, None] / Ly)
    u = np.zeros(g.shape2())
    v = np.zeros(g.shape2())
    u[1:, :] = -(psi[1:, :] - psi[:-1, :]) / dx
    v[:, 1:] = (psi[:, 1:] - psi[:, :-1]) / dx
    u *= (au == 1)
    v *= (av == 1)
    scale = umax / max(np.abs(u).max(), np.abs(v).max(), 1e-300)
    u *= scale
    v *= scale
    shp = g.shape3()
    hh = np.full(shp, h)
    hh[0] = 0.0
    uu = np.zeros(shp)
    vv = np.zeros(shp)
    lay = 1.0 + shear * ((np.arange(1, kmax + 1) - 0.5) / kmax - 0.5)
    uu[1:] = u[None] * h * lay[:, None, None]
    vv[1:] = v[None] * h * lay[:, None, None]
    xT = (i - g.imin + 0.5) * dx
    yT = (j - g.jmin + 0.5) * dx
    s = sigma_cells * dx
    blob = np.exp(-((xT[None, :] - Lx / 2) ** 2 + (yT[:, None] - Ly / 2) ** 2) / (2 * s * s))
    f = np.zeros(shp)
    prof = 1.0 + vertical * np.cos(np.pi * (np.arange(1, kmax + 1) - 0.5) / kmax)
    f[1:] = blob[None] * prof[:, None, None]
    f[1:] += slope * (xT[None, None, :] / Lx + yT[None, :, None] / Ly)
    f[1:] += rng.uniform(-noise, noise, size=(kmax, g.nj, g.ni))
    f *= (az >= 1)[None]
    c = Case(g, az=az, au=au, av=av, ax=ax, f=f.astype(dtype), uu=uu.astype(dtype), vv=vv.astype(dtype),
             ww=np.zeros(shp, dtype), ho=hh.astype(dtype), hn=hh.copy().astype(dtype),
             hun=hh.copy().astype(dtype), hvn=hh.copy().astype(dtype), nuh=np.full(shp, nuh, dtype=dtype))
    c.par.update(dt=dt, split=2, hscheme=4, vscheme=4, AH=0.0, cnpar=1.0, avmol=0.0, adv_ver_iterations=1)
    return c


def box_weights(case: Case, box=32):
    """dJ/df for J = tracer content of a centred box x box column block, all levels:
    J = sum f * hn / ard1 over its wet cells (k = 1..kmax)."""
    g = case.grid
    w = np.zeros(g.shape3())
    j0 = HALO + (g.ny - box) // 2
    i0 = HALO + (g.nx - box) // 2
    sl = (slice(1, None), slice(j0, j0 + box), slice(i0, i0 + box))
    w[sl] = case["hn"][sl] / g.ard1
    w *= (case["az"] == 1)[None]
    return w


def random_case(nx=24, ny=20, kmax=7, seed=0, dtype=np.float64, land=0.2, open_bdy=True, dx=400.0, dy=300.0,
                dt=30.0, cfl=0.8, wscale=0.5) -> Case:
    """Random fields over a random mask for routine-level parity tests.

    az: 1 on random interior cells (fraction ~1-land), 0 on land and in the halo; with
    open_bdy a stretch of the western and southern interior edges is set to 2 (open-boundary
    cells, domain.F90:269-286) so that the au/av values 2 and 3 occur. Velocities are scaled
    so that the horizontal Courant numbers stay below `cfl`; ww has w(0) = w(kmax) = 0.
    """
    g = Grid(nx, ny, kmax, dx, dy)
    rng = np.random.default_rng(seed)
    az = np.zeros(g.shape2(), np.int32)
    inner = (rng.random((ny, nx)) > land).astype(np.int32)
    az[g.interior()] = inner
    if open_bdy:
        jj = slice(HALO + ny // 4, HALO + ny // 4 + max(2, ny // 3))
        az[jj, HALO] = 2
        ii = slice(HALO + nx // 3, HALO + nx // 3 + max(2, nx // 3))
        az[HALO, ii] = 2
    au, av, ax = derive_uvx(az)
    shp = g.shape3()
    ho = rng.uniform(0.5, 2.0, shp)
    hn = rng.uniform(0.5, 2.0, shp)
    hun = rng.uniform(0.5, 2.0, shp)
    hvn = rng.uniform(0.5, 2.0, shp)
    # transports: |uu|/hun*dt/dx < cfl
    uu = rng.uniform(-1, 1, shp) * hun * cfl * dx / dt * 0.5
    vv = rng.uniform(-1, 1, shp) * hvn * cfl * dy / dt * 0.5
    ww = rng.uniform(-1, 1, shp) * wscale * 0.5 / dt  # |w|*dt/h < ~0.5
    ww[0] = 0.0
    ww[kmax] = 0.0
    f = rng.normal(size=shp)
    nuh = rng.uniform(1e-5, 1e-2, shp)
    c = Case(g, az=az, au=au, av=av, ax=ax, f=f.astype(dtype), uu=uu.astype(dtype), vv=vv.astype(dtype),
             ww=ww.astype(dtype), ho=ho.astype(dtype), hn=hn.astype(dtype), hun=hun.astype(dtype),
             hvn=hvn.astype(dtype), nuh=nuh.astype(dtype))
    c.par.update(dt=dt)
    return c
