"""Module state of the mode-split step (variables_2d / variables_3d / domain of the reference)
as one table of fields, plus seeded synthetic baroclinic cases.

The order of the name lists is part of the C ABI (getm_bc_state in include/getm_b200.h; the
oracle keeps the same order): F2_NAMES are the 2D fields (always FP64), F3_NAMES the 3D fields
(FP64, or FP32 in the mixed-precision variant), PD/PI the real and integer parameters.
"""
from __future__ import annotations

import math

import numpy as np

from .cases import derive_uvx
from .grid import HALO, Grid

F2_NAMES = ["z", "zo", "U", "V", "D", "DU", "DV", "UEx", "VEx", "fU", "fV", "ru", "rv", "ruu", "rvv", "Uint", "Vint",
            "Uinto", "Vinto", "SlUx", "SlVx", "Slru", "Slrv", "zub", "zvb", "zub0", "zvb0", "fwf", "H", "HU", "HV",
            "dry_z", "dry_u", "dry_v", "coru", "corv", "tausx", "tausy", "airp", "sseo", "ssen", "ssuo", "ssun",
            "ssvo", "ssvn", "Dn", "Dun", "Dvn", "rru", "rrv", "taubx", "tauby", "taub", "taus",
            "swr", "shf", "A", "g1", "g2"]
F3_NAMES = ["uu", "vv", "ww", "ho", "hn", "huo", "hun", "hvo", "hvn", "uuEx", "vvEx", "idpdx", "idpdy", "T", "S",
            "rho", "buoy", "num", "nuh", "rad", "tke", "eps", "Tlo", "Slo"]
PD_NAMES = ["dtm", "dt", "cnpar", "min_depth", "crit_depth", "g", "rho_0", "kappa", "avmmol", "avmolt", "avmols", "T0",
            "S0", "dtr0", "dsr0", "ip_fac", "temp_AH", "salt_AH", "avmback", "avhback", "cp", "swr_bot_refl_frac",
            "swr_min_bot_frac"]
PI_NAMES = ["M", "MM", "runtype", "vel2d_adv_split", "vel2d_adv_hor", "vel3d_adv_split", "vel3d_adv_hor",
            "vel3d_adv_ver", "temp_adv_split", "temp_adv_hor", "temp_adv_ver", "salt_adv_split", "salt_adv_hor",
            "salt_adv_ver", "adv_ver_iterations", "ufirst2d", "ufirst3d", "calc_temp", "calc_salt", "ip_method",
            "viscosity", "eqstate_method", "sealevel_check", "radiation", "nan_warned"]
# fields that only a switched-on option reads or writes (radiation: swr, shf, A, g1, g2, rad;
# PARABOLIC_VISCOSITY: tke, eps, each optional; the mixed step's compensated storage of T and S:
# Tlo, Slo): a device state may leave them out (NULL)
OPTIONAL_F2 = ("swr", "shf", "A", "g1", "g2")
OPTIONAL_F3 = ("rad", "tke", "eps", "Tlo", "Slo")
# values of the parameters added after the first fixtures were written (their defaults in the
# reference: variables_3d.F90:120, parameters.F90:23, temperature.F90:50-51, m2d.F90:82,
# eqstate.F90:27 -- where the configurations use the linear equation of state)
PARAM_DEFAULTS_PD = dict(avmback=0.0, avhback=0.0, cp=3985.0, swr_bot_refl_frac=-1.0,
                         swr_min_bot_frac=float(np.float32(0.01)))
PARAM_DEFAULTS_PI = dict(ip_method=1, viscosity=0, eqstate_method=1, sealevel_check=0, radiation=0, nan_warned=0)

F32 = lambda x: float(np.float32(x))  # noqa: E731  -- a Fortran default-kind real literal widened to double

# parameters.F90:21-27 and eqstate.F90:27 literals are single precision in the reference
DEFAULT_PD = dict(g=F32(9.81), rho_0=1025.0, kappa=F32(0.4), avmmol=F32(1.8e-6), avmolt=F32(1.4e-7),
                  avmols=F32(1.1e-9), T0=10.0, S0=33.75, dtr0=F32(-0.17), dsr0=F32(0.78), ip_fac=1.0, temp_AH=-1.0,
                  salt_AH=-1.0, cnpar=F32(0.9), min_depth=0.5, crit_depth=2.0, avmback=0.0, avhback=0.0, cp=3985.0,
                  swr_bot_refl_frac=-1.0, swr_min_bot_frac=F32(0.01))
P2_PDM, HALFSPLIT = 6, 2


# 2D open-boundary types (cppdefs.h:65-68)
ZERO_GRADIENT, SOMMERFELD, CLAMPED, FLATHER_ELEV = 1, 2, 3, 4


class OpenBoundaries:
    """Open-boundary segments of a domain (bdy_spec.F90) and their elevation data.

    Each side is a list of (pos, first, last, type2d): western (wi, wfj, wlj), northern
    (nj, nfi, nli), eastern (ei, efj, elj), southern (sj, sfi, sli), reference indices. The
    boundary points are numbered in segment order W, N, E, S (bdy_map). Elevation data: either a
    fixed `data` array per point (plus `data_u` / `data_v` for FLATHER_ELEV), or harmonic,
    amp*sin(2*pi*loop*dtm/period + phase) per point at micro step `loop`.
    """

    def __init__(self, west=(), north=(), east=(), south=(), ramp=-1, amp=None, phase=None, period=0.0,
                 data=None, data_u=None, data_v=None):
        self.sides = [list(west), list(north), list(east), list(south)]
        self.ramp = int(ramp)
        n = self.npoints()
        self.amp = None if amp is None else np.broadcast_to(np.asarray(amp, np.float64), (n,)).copy()
        self.phase = (None if amp is None else
                      np.broadcast_to(np.asarray(0.0 if phase is None else phase, np.float64), (n,)).copy())
        self.period = float(period)
        self.data = None if data is None else np.asarray(data, np.float64).copy()
        self.data_u = None if data_u is None else np.asarray(data_u, np.float64).copy()
        self.data_v = None if data_v is None else np.asarray(data_v, np.float64).copy()

    def segments(self):
        return [seg for side in self.sides for seg in side]

    def npoints(self):
        return sum(last - first + 1 for (_, first, last, _) in self.segments())

    def struct(self):
        """ctypes struct of the C layout getm_bdy (include/getm_b200.h); keeps its arrays alive."""
        import ctypes as C

        segs = self.segments()
        self._seg = np.array([[p, f, l] for (p, f, l, _) in segs], np.int32).reshape(-1)
        self._typ = np.array([t for (_, _, _, t) in segs], np.int32)
        b = GetmBdy()
        b.nwb, b.nnb, b.neb, b.nsb = (len(x) for x in self.sides)
        b.seg = self._seg.ctypes.data if len(segs) else None
        b.type2d = self._typ.ctypes.data if len(segs) else None
        b.ramp = self.ramp
        b.npoints = self.npoints()
        for name in ("data", "data_u", "data_v", "amp", "phase"):
            a = getattr(self, name)
            setattr(b, name, None if a is None else a.ctypes.data)
        b.period = self.period
        return b


def _bdy_struct_type():
    import ctypes as C

    class _GetmBdy(C.Structure):
        _fields_ = [("nwb", C.c_int32), ("nnb", C.c_int32), ("neb", C.c_int32), ("nsb", C.c_int32),
                    ("seg", C.c_void_p), ("type2d", C.c_void_p), ("ramp", C.c_int32), ("npoints", C.c_int32),
                    ("data", C.c_void_p), ("data_u", C.c_void_p), ("data_v", C.c_void_p), ("amp", C.c_void_p),
                    ("phase", C.c_void_p), ("period", C.c_double)]

    return _GetmBdy


GetmBdy = _bdy_struct_type()


class BcCase:
    """A full model state (numpy arrays in the reference layout) with parameters."""

    def __init__(self, grid: Grid, dtype3=np.float64, alloc3=True):
        self.grid = grid
        self.dtype3 = np.dtype(dtype3)
        self.f2 = {n: np.zeros(grid.shape2()) for n in F2_NAMES}
        self.f3 = {n: np.zeros(grid.shape3(), dtype=self.dtype3) for n in F3_NAMES} if alloc3 else {}
        self.az = self.au = self.av = self.ax = None
        self.pd = {n: 0.0 for n in PD_NAMES}
        self.pi = {n: 0 for n in PI_NAMES}
        self.pi["ip_method"] = 1  # internal_pressure.F90:80 (BLUMBERG_MELLOR)
        self.pi["eqstate_method"] = 1  # linear, as the configurations ask
        self.bdy = None  # OpenBoundaries, or None for a closed domain

    def copy(self, dtype3=None):
        c = BcCase(self.grid, dtype3 or self.dtype3)
        c.f2 = {k: v.copy() for k, v in self.f2.items()}
        c.f3 = {k: v.astype(c.dtype3) for k, v in self.f3.items()}
        c.az, c.au, c.av, c.ax = self.az.copy(), self.au.copy(), self.av.copy(), self.ax.copy()
        c.pd, c.pi = dict(self.pd), dict(self.pi)
        c.bdy = self.bdy
        return c

    def masks(self):
        return self.az, self.au, self.av, self.ax


def _eqstate(c: BcCase):
    p = c.pd
    T, S = c.f3["T"].astype(np.float64), c.f3["S"].astype(np.float64)
    rho = p["rho_0"] + p["dtr0"] * (T - p["T0"]) + p["dsr0"] * (S - p["S0"])
    rho[0] = 0.0
    buoy = (-p["g"] / p["rho_0"]) * (rho - p["rho_0"])
    buoy[0] = 0.0
    c.f3["rho"][...] = rho
    c.f3["buoy"][...] = buoy


def baroclinic_case(nx=32, ny=24, kmax=8, recipe="shelf", dx=1000.0, M=20, dt3=60.0, seed=2, dtype3=np.float64,
                    land=0.0, hmin=5.0, hmax=150.0, nu_max=1e-2, latitude=54.0, bdy=None, t_background=15.0,
                    t_noise=0.0) -> BcCase:
    """Seeded initial state of the mode-split step, closed basin.

    recipe 'shelf': H = 10 + 190*0.5*(1+tanh((x-x0)/L)), L = 20 cells, x0 = nx/2.
    recipe 'flat':  H = 20 m.
    recipe 'rotation': H = 20 m, solid-body rotation and a temperature anomaly (see _rotation_start)
      of 1 C on t_background, plus seeded uniform noise of amplitude t_noise.
    recipe 'islands': H = hmin + (hmax-hmin)*(field-p)/(max-p) on wet cells of a Gaussian-smoothed
      noise field (sigma = 40 cells, scaled with the grid), land where field < its `land` quantile.
    Stratification: T from 20 C (surface) to 8 C (bottom) linear in depth plus N(0, 0.1) noise,
    S from 30 to 35 psu; linear EOS. Viscosity / diffusivity: static parabolic 4*nu_max*s*(1-s)
    (+1e-6) over the sigma levels. Coriolis on an f-plane at `latitude` (domain.F90:364-369 with the
    reference's single-precision omega = 2*pi/86164).
    bdy: OpenBoundaries; its segment points become boundary points (az = 2, domain.F90:263-280).
    """
    c, rng = _baroclinic_2d(nx, ny, kmax, recipe, dx, M, dt3, seed, dtype3, land, hmin, hmax, latitude, True, bdy)
    _baroclinic_3d_numpy(c, rng, nu_max)
    if recipe == "rotation":
        _rotation_start(c, background=t_background, noise=t_noise, seed=seed)
    return c


def _rotation_start(c: BcCase, umax=0.5, sigma_cells=8.0, background=15.0, noise=0.0, seed=3):
    """recipe 'rotation' (flat 20 m): solid-body rotation of the whole water column (the discrete
    curl of psi = 0.5*omega*min(r,R)^2 at X points, R = nx/2 cells, omega = umax/R; depth-uniform
    velocity, so uu = u*hun, U = sum of uu) and a temperature anomaly of 1 C (Gaussian, sigma =
    sigma_cells) on `background` C at (0.3 nx, 0.5 ny), plus uniform noise in [-noise, noise]
    (numpy default_rng(seed + 1000)); S = 35."""
    g = c.grid
    f2, f3 = c.f2, c.f3
    dx = g.dx
    i = np.arange(g.imin - HALO, g.imax + HALO + 1)
    j = np.arange(g.jmin - HALO, g.jmax + HALO + 1)
    xX, yX = (i - g.imin + 1) * dx, (j - g.jmin + 1) * dx
    xc, yc, R = g.nx * dx / 2, g.ny * dx / 2, (g.nx / 2) * dx
    om = umax / R
    r = np.sqrt((xX[None, :] - xc) ** 2 + (yX[:, None] - yc) ** 2)
    psi = 0.5 * om * np.minimum(r, R) ** 2
    u = np.zeros(g.shape2())
    v = np.zeros(g.shape2())
    u[1:, :] = -(psi[1:, :] - psi[:-1, :]) / dx
    v[:, 1:] = (psi[:, 1:] - psi[:, :-1]) / dx
    u *= (c.au == 1)
    v *= (c.av == 1)
    uu = u[None] * f3["hun"].astype(np.float64)
    vv = v[None] * f3["hvn"].astype(np.float64)
    uu[0] = 0.0
    vv[0] = 0.0
    f3["uu"][...] = uu
    f3["vv"][...] = vv
    f2["U"][...] = uu[1:].sum(axis=0)
    f2["V"][...] = vv[1:].sum(axis=0)
    xT, yT = (i - g.imin + 0.5) * dx, (j - g.jmin + 0.5) * dx
    s = sigma_cells * dx
    blob = np.exp(-((xT[None, :] - 0.3 * g.nx * dx) ** 2 + (yT[:, None] - 0.5 * g.ny * dx) ** 2) / (2 * s * s))
    wet3 = (c.az >= 1)[None]
    T = background + blob[None] + np.zeros(g.shape3())
    if noise > 0:
        T = T + np.random.default_rng(seed + 1000).uniform(-noise, noise, g.shape3())
    S = np.full(g.shape3(), 35.0)
    T[0] = 0.0
    S[0] = 0.0
    f3["T"][...] = np.where(wet3, T, 0.0)
    f3["S"][...] = np.where(wet3, S, 0.0)
    _eqstate(c)


def _baroclinic_2d(nx, ny, kmax, recipe, dx, M, dt3, seed, dtype3, land, hmin, hmax, latitude, alloc3, bdy=None):
    """The 2D part of :func:`baroclinic_case` (masks, depths, elevations, parameters)."""
    g = Grid(nx, ny, kmax, dx, dx)
    rng = np.random.default_rng(seed)
    c = BcCase(g, dtype3, alloc3=alloc3)
    i = np.arange(g.imin - HALO, g.imax + HALO + 1)
    xT = (i - g.imin + 0.5) * dx
    az = np.zeros(g.shape2(), np.int32)
    if recipe == "shelf":
        L = 20 * dx
        x0 = nx / 2 * dx
        H = np.broadcast_to(10.0 + 190.0 * 0.5 * (1.0 + np.tanh((xT - x0) / L)), g.shape2()).copy()
        az[g.interior()] = 1
    elif recipe in ("flat", "rotation"):
        H = np.full(g.shape2(), 20.0)
        az[g.interior()] = 1
    elif recipe == "islands":
        field = rng.normal(size=(ny, nx))
        sig = max(1.0, 40.0 * nx / 2048.0)
        k1 = np.fft.fftfreq(nx)[None, :]
        k2 = np.fft.fftfreq(ny)[:, None]
        field = np.real(np.fft.ifft2(np.fft.fft2(field) * np.exp(-2 * (math.pi * sig) ** 2 * (k1 ** 2 + k2 ** 2))))
        field = (field - field.mean()) / field.std()
        p = np.quantile(field, land) if land > 0 else field.min() - 1e-9
        wet = field >= p
        Hi = np.where(wet, hmin + (hmax - hmin) * (field - p) / (field.max() - p), 0.0)
        H = np.zeros(g.shape2())
        H[g.interior()] = Hi
        az[g.interior()] = wet.astype(np.int32)
        # halo depths mirror the first interior line (update_2d_halo with mirror, halo_zones.F90:110-118)
        H[:, 1] = H[:, 2]; H[:, -2] = H[:, -3]; H[1, :] = H[2, :]; H[-2, :] = H[-3, :]  # noqa: E702
    else:
        raise ValueError(recipe)
    if recipe != "islands":
        H[:, 1] = H[:, 2]; H[:, -2] = H[:, -3]; H[1, :] = H[2, :]; H[-2, :] = H[-3, :]  # noqa: E702
        H[:, 0] = H[:, 1]; H[:, -1] = H[:, -2]; H[0, :] = H[1, :]; H[-1, :] = H[-2, :]  # noqa: E702
    if bdy is not None:
        def ix(i, j):
            return j - (g.jmin - HALO), i - (g.imin - HALO)
        for side, segs in enumerate(bdy.sides):
            for (pos, first, last, _) in segs:
                for q in range(first, last + 1):
                    az[ix(pos, q) if side in (0, 2) else ix(q, pos)] = 2
        c.bdy = bdy
    au, av, ax = derive_uvx(az)
    c.az, c.au, c.av, c.ax = az, au, av, ax
    f2 = c.f2
    f2["H"][...] = H
    # uv_depths vel_depth_method = 0 (uv_depths.F90: HU = 0.5*(H(i)+H(i+1)))
    f2["HU"][:, :-1] = 0.5 * (H[:, :-1] + H[:, 1:])
    f2["HV"][:-1, :] = 0.5 * (H[:-1, :] + H[1:, :])
    p = c.pd
    p.update(DEFAULT_PD)
    dtm = dt3 / M
    p.update(dtm=dtm, dt=dt3)
    c.pi.update(M=M, MM=1, runtype=4, vel2d_adv_split=HALFSPLIT, vel2d_adv_hor=P2_PDM, vel3d_adv_split=HALFSPLIT,
                vel3d_adv_hor=P2_PDM, vel3d_adv_ver=P2_PDM, temp_adv_split=HALFSPLIT, temp_adv_hor=P2_PDM,
                temp_adv_ver=P2_PDM, salt_adv_split=HALFSPLIT, salt_adv_hor=P2_PDM, salt_adv_ver=P2_PDM,
                adv_ver_iterations=1, ufirst2d=0, ufirst3d=1, calc_temp=1, calc_salt=1)
    pi_ = F32(3.141592654)
    omega = 2.0 * pi_ / F32(86164.0)
    cori = 2.0 * omega * math.sin(pi_ / 180.0 * latitude)
    f2["coru"][...] = cori * (au > 0)
    f2["corv"][...] = cori * (av > 0)
    f2["zub0"][...] = 0.01
    f2["zvb0"][...] = 0.01
    f2["zub"][...] = 0.01
    f2["zvb"][...] = 0.01
    # elevation: small seeded perturbation on wet points; depths from depth_update
    z = np.zeros(g.shape2())
    wet = az >= 1
    z[wet] = 0.05 * rng.normal(size=int(wet.sum()))
    f2["z"][...] = z
    f2["zo"][...] = z
    zo = z
    D = z + H
    f2["D"][...] = D
    xu = np.maximum(0.25 * (zo[:, :-1] + zo[:, 1:] + z[:, :-1] + z[:, 1:]), -f2["HU"][:, :-1] + p["min_depth"])
    f2["DU"][:, :-1] = xu + f2["HU"][:, :-1]
    xv = np.maximum(0.25 * (zo[:-1, :] + zo[1:, :] + z[:-1, :] + z[1:, :]), -f2["HV"][:-1, :] + p["min_depth"])
    f2["DV"][:-1, :] = xv + f2["HV"][:-1, :]
    d1 = 2 * p["min_depth"]
    d2i = 1.0 / (p["crit_depth"] - 2 * p["min_depth"])
    f2["dry_z"][...] = np.where(az > 0, np.clip((D - 0.5 * d1) * d2i, 0, 1), 0.0)
    f2["dry_u"][...] = np.where(au > 0, np.clip((f2["DU"] - d1) * d2i, 0, 1), 0.0)
    f2["dry_v"][...] = np.where(av > 0, np.clip((f2["DV"] - d1) * d2i, 0, 1), 0.0)
    # macro-step elevations: old = new = z (start-up)
    for a, b in (("sseo", "z"), ("ssen", "z")):
        f2[a][...] = f2[b]
    ssu = np.zeros(g.shape2())
    ssu[:, :-1] = np.maximum(0.5 * (z[:, :-1] + z[:, 1:]), -f2["HU"][:, :-1] + p["min_depth"])
    ssv = np.zeros(g.shape2())
    ssv[:-1, :] = np.maximum(0.5 * (z[:-1, :] + z[1:, :]), -f2["HV"][:-1, :] + p["min_depth"])
    f2["ssuo"][...] = ssu
    f2["ssun"][...] = ssu
    f2["ssvo"][...] = ssv
    f2["ssvn"][...] = ssv
    f2["Dn"][...] = f2["ssen"] + H
    f2["Dun"][...] = f2["ssun"] + f2["HU"]
    f2["Dvn"][...] = f2["ssvn"] + f2["HV"]
    return c, rng


def _profiles(kmax, nu_max):
    """1D vertical profiles: depth fraction of layer centres (0 at the surface, 1 at the bottom)
    and the parabolic viscosity at the interfaces."""
    sig = (np.arange(kmax + 1) - 0.5) / kmax
    depth_frac = 1.0 - sig
    s = np.arange(kmax + 1) / kmax
    nu = 4 * nu_max * s * (1 - s) + 1e-6
    return depth_frac, nu


def _baroclinic_3d_numpy(c: BcCase, rng, nu_max):
    g = c.grid
    kmax = g.kmax
    f2 = c.f2
    H = f2["H"]
    az = c.az
    # layer heights (sigma_coordinates, all levels)
    f3 = c.f3
    f3["ho"][...] = ((f2["sseo"] + H) / kmax)[None]
    f3["hn"][...] = ((f2["ssen"] + H) / kmax)[None]
    f3["huo"][...] = ((f2["ssuo"] + f2["HU"]) / kmax)[None]
    f3["hun"][...] = ((f2["ssun"] + f2["HU"]) / kmax)[None]
    f3["hvo"][...] = ((f2["ssvo"] + f2["HV"]) / kmax)[None]
    f3["hvn"][...] = ((f2["ssvn"] + f2["HV"]) / kmax)[None]
    # stratification on sigma levels: depth of layer centre
    depth_frac, nu = _profiles(kmax, nu_max)
    depth_frac = depth_frac[:, None, None]
    T = 20.0 - 12.0 * depth_frac + 0.1 * rng.normal(size=g.shape3())
    S = 30.0 + 5.0 * depth_frac + np.zeros(g.shape3())
    T[0] = 0.0
    S[0] = 0.0
    wet3 = (az >= 1)[None]
    f3["T"][...] = np.where(wet3, T, 0.0)
    f3["S"][...] = np.where(wet3, S, 0.0)
    # viscosity / diffusivity at interfaces k (between layers k and k+1): sigma_k = k/kmax
    f3["num"][...] = nu[:, None, None]
    f3["nuh"][...] = nu[:, None, None]
    _eqstate(c)


def baroclinic_case_device(nx=2048, ny=2048, kmax=50, recipe="islands", dx=1000.0, M=20, dt3=60.0, seed=6,
                           dtype3=None, land=0.3, hmin=5.0, hmax=150.0, nu_max=1e-2, latitude=54.0, device="cuda",
                           compensated=True):
    """:func:`baroclinic_case` with the 3D fields built on the device (for the 2048 x 2048 x 50
    domain, whose 19 FP64 3D fields would take ~33 GB of host memory). 2D fields and parameters
    are computed in numpy exactly as in baroclinic_case; the temperature noise comes from a seeded
    device generator. Returns a code_b200.getm.BcDevice."""
    import torch

    from .getm import BcDevice

    dtype3 = dtype3 or torch.float64
    c, _ = _baroclinic_2d(nx, ny, kmax, recipe, dx, M, dt3, seed, np.float64, land, hmin, hmax, latitude, False)
    g = c.grid
    kmax = g.kmax
    t = {}
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    for n in F2_NAMES:
        t["f2_" + n] = dev(c.f2[n])
    for n, m in zip(("az", "au", "av", "ax"), c.masks()):
        t[n] = dev(m)
    f2 = c.f2
    shp = g.shape3()
    ones = torch.ones((kmax + 1, 1, 1), dtype=torch.float64, device=device)

    def level_const(a2):
        return (ones * dev(a2)[None]).to(dtype3).contiguous()

    t["f3_ho"] = level_const((f2["sseo"] + f2["H"]) / kmax)
    t["f3_hn"] = level_const((f2["ssen"] + f2["H"]) / kmax)
    t["f3_huo"] = level_const((f2["ssuo"] + f2["HU"]) / kmax)
    t["f3_hun"] = level_const((f2["ssun"] + f2["HU"]) / kmax)
    t["f3_hvo"] = level_const((f2["ssvo"] + f2["HV"]) / kmax)
    t["f3_hvn"] = level_const((f2["ssvn"] + f2["HV"]) / kmax)
    depth_frac, nu = _profiles(kmax, nu_max)
    dfr = dev(depth_frac)[:, None, None]
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    wet = dev((c.az >= 1).astype(np.float64))[None]
    T = (20.0 - 12.0 * dfr + 0.1 * torch.randn(shp, generator=gen, device=device, dtype=torch.float64)) * wet
    S = (30.0 + 5.0 * dfr + torch.zeros(shp, dtype=torch.float64, device=device)) * wet
    T[0] = 0.0
    S[0] = 0.0
    p = c.pd
    rho = p["rho_0"] + p["dtr0"] * (T - p["T0"]) + p["dsr0"] * (S - p["S0"])
    rho[0] = 0.0
    buoy = (-p["g"] / p["rho_0"]) * (rho - p["rho_0"])
    buoy[0] = 0.0
    t["f3_T"], t["f3_S"], t["f3_rho"], t["f3_buoy"] = (x.to(dtype3).contiguous() for x in (T, S, rho, buoy))
    nuv = dev(nu)[:, None, None] * torch.ones(shp, dtype=torch.float64, device=device)
    t["f3_num"] = nuv.to(dtype3).contiguous()
    t["f3_nuh"] = nuv.to(dtype3).contiguous()
    for n in ("uu", "vv", "ww", "uuEx", "vvEx", "idpdx", "idpdy"):
        t["f3_" + n] = torch.zeros(shp, dtype=dtype3, device=device)
    if dtype3 == torch.float32 and compensated:  # the mixed step's compensated storage of T and S
        t["f3_Tlo"] = torch.zeros(shp, dtype=torch.float16, device=device)
        t["f3_Slo"] = torch.zeros(shp, dtype=torch.float16, device=device)
    return g, BcDevice(tensors=t, pd=dict(c.pd), pi=dict(c.pi))


# -------------------------------------------------------------------------------------------------
def oracle_struct(c: BcCase):
    """ctypes struct (or_bc) of numpy pointers for the oracle; keeps references alive."""
    import ctypes as C

    from .grid import HALO as _  # noqa: F401

    n2, n3, npd, npi = len(F2_NAMES), len(F3_NAMES), len(PD_NAMES), len(PI_NAMES)

    class OrBc(C.Structure):
        _fields_ = [("f2", C.c_void_p * n2), ("f3", C.c_void_p * n3), ("az", C.c_void_p), ("au", C.c_void_p),
                    ("av", C.c_void_p), ("ax", C.c_void_p), ("par", C.c_double * npd), ("ipar", C.c_int * npi),
                    ("bdy", C.c_void_p)]

    s = OrBc()
    for q, nm in enumerate(F2_NAMES):
        a = c.f2[nm]
        assert a.flags.c_contiguous and a.dtype == np.float64
        s.f2[q] = a.ctypes.data
    for q, nm in enumerate(F3_NAMES):
        a = c.f3[nm]
        assert a.flags.c_contiguous and a.dtype == c.dtype3
        s.f3[q] = a.ctypes.data
    s.az, s.au, s.av, s.ax = (m.ctypes.data for m in c.masks())
    for q, nm in enumerate(PD_NAMES):
        s.par[q] = c.pd[nm]
    for q, nm in enumerate(PI_NAMES):
        s.ipar[q] = int(c.pi[nm])
    if c.bdy is not None:
        s._bdy = c.bdy.struct()
        s.bdy = C.addressof(s._bdy)
    return s


def read_back_ipar(c: BcCase, s):
    for q, nm in enumerate(PI_NAMES):
        c.pi[nm] = int(s.ipar[q])
