"""Generates tests/golden/reference_mode_split.npz: the reference's own integrate_2d / integrate_3d
(the mode-split time loop, integration.F90:98-172) executed from source (fortran_subset.py) on a
small closed basin, together with the inputs. The oracle and the CUDA path are compared with it
bit for bit (tests/test_golden_bc_cpu.py) and the CUDA path within 1e-12 (tests/test_gpu_baroclinic.py).

    python tests/golden/make_golden_bc.py [closed] [bdy] [ip2] ... [ip7] [phys3] [phys2] [nan] [hotstart]

Configuration: runtype 4 (prognostic T and S), sigma coordinates (equidistant), linear equation of
state, Blumberg-Mellor internal pressure (reference_mode_split_ip2.npz: the linear Blumberg-Mellor
variant, Song-Wright and Chu-Fan -- ip_method 2, 4, 5 -- in reference_mode_split_ip{2,4,5}.npz on an
islands basin; see ip_case()), P2_PDM / HALFSPLIT advection of momentum (2D and 3D) and
tracers, closed boundaries, num/nuh prescribed (the turbulence closure -- the un-vendored GOTM -- is
replaced by a routine that leaves them unchanged; ss_nn, whose outputs only feed it, likewise),
no wind, air pressure, freshwater or short-wave forcing. The second fixture,
reference_mode_split_bdy.npz, adds open boundaries of all four 2D types (update_2d_bdy.F90,
mirror_bdy_2d.F90, mirror_bdy_3d.F90); see bdy_case().
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

import fortran_subset as fs  # noqa: E402
from code_b200 import state as S  # noqa: E402

FILES = [
    "src/futils/tridiagonal.F90", "src/2d/advection.F90", "src/2d/adv_split_u.F90", "src/2d/adv_split_v.F90",
    "src/3d/advection_3d.F90", "src/3d/adv_split_w.F90",
    "src/2d/bottom_friction.F90", "src/2d/uv_advect.F90", "src/2d/uv_diffusion.F90", "src/2d/momentum.F90",
    "src/2d/sealevel.F90", "src/2d/depth_update.F90", "src/domain/mirror_bdy_2d.F90", "src/domain/mirror_bdy_3d.F90",
    "src/3d/start_macro.F90", "src/3d/stop_macro.F90", "src/3d/bottom_friction_3d.F90",
    "src/3d/internal_pressure.F90", "src/3d/ip_blumberg_mellor.F90", "src/3d/ip_blumberg_mellor_lin.F90",
    "src/3d/ip_z_interpol.F90", "src/3d/ip_song_wright.F90", "src/3d/ip_chu_fan.F90",
    "src/3d/ip_shchepetkin_mcwilliams.F90", "src/3d/ip_stelling_vankester.F90",
    "src/3d/uu_momentum_3d.F90",
    "src/3d/vv_momentum_3d.F90", "src/3d/coordinates.F90", "src/3d/sigma_coordinates.F90",
    "src/3d/ww_momentum_3d.F90", "src/3d/uv_advect_3d.F90", "src/3d/uv_diffusion_3d.F90", "src/3d/stresses_3d.F90",
    "src/3d/temperature.F90", "src/3d/salinity.F90", "src/3d/eqstate.F90", "src/3d/slow_bottom_friction.F90",
    "src/3d/slow_terms.F90", "src/2d/m2d.F90", "src/3d/m3d.F90", "src/2d/update_2d_bdy.F90",
]


class RefBc:
    def __init__(self, c: S.BcCase):
        self.c = c
        g = self.g = c.grid
        # PARABOLIC_VISCOSITY is a compile-time option of the reference (gotm.F90:131, m3d.F90:571)
        P = self.P = fs.Program(defines=("PARABOLIC_VISCOSITY",) if c.pi.get("viscosity", 0) == 1 else ())
        F2, F3 = self.F2, self.F3
        f2 = {k.lower(): F2(v) for k, v in c.f2.items()}
        f3 = {k.lower(): F3(v) for k, v in c.f3.items()}
        self.f2, self.f3 = f2, f3
        zero2 = lambda: F2(np.zeros(g.shape2()))  # noqa: E731
        zero3 = lambda: F3(np.zeros(g.shape3()))  # noqa: E731
        pd, pi = c.pd, c.pi
        P.add_module_namespace("parameters", g=pd["g"], rho_0=pd["rho_0"], cp=np.float64(pd["cp"]),
                               kappa=pd["kappa"], avmmol=pd["avmmol"], avmolt=pd["avmolt"], avmols=pd["avmols"])
        P.add_module_namespace(
            "domain", imin=g.imin, imax=g.imax, jmin=g.jmin, jmax=g.jmax, kmax=g.kmax, ioff=0, joff=0, dx=g.dx,
            dy=g.dy, ard1=g.ard1, az=F2(c.az), au=F2(c.au), av=F2(c.av), ax=F2(c.ax), h=f2["h"], hu=f2["hu"],
            hv=f2["hv"], min_depth=pd["min_depth"], crit_depth=pd["crit_depth"], dry_z=f2["dry_z"],
            dry_u=f2["dry_u"], dry_v=f2["dry_v"], cori=zero2(), coru=f2["coru"], corv=f2["corv"],
            ga=None, ddu=np.float64(0.0), ddl=np.float64(0.0), vert_cord=1, maxdepth=np.float64(0.0), z0_method=0,
            z0_const=np.float64(0.01), z0=zero2(), ill=g.imin, ihl=g.imax, jll=g.jmin, jhl=g.jmax, ilg=g.imin,
            ihg=g.imax, jlg=g.jmin, jhg=g.jmax, **self._bdy_domain(c.bdy))
        v2 = {k: f2[k] for k in ("z", "zo", "u", "v", "d", "du", "dv", "uex", "vex", "fu", "fv", "ru", "rv", "ruu",
                                 "rvv", "uint", "vint", "uinto", "vinto", "slux", "slvx", "slru", "slrv", "zub",
                                 "zvb", "zub0", "zvb0", "fwf")}
        v2["fwf_int"] = zero2()
        P.add_module_namespace("variables_2d", **v2)
        v3 = {k: f3[k] for k in ("uu", "vv", "ww", "ho", "hn", "huo", "hun", "hvo", "hvn", "uuex", "vvex", "idpdx",
                                 "idpdy", "t", "s", "rho", "buoy", "num", "nuh")}
        v3["s"] = f3["s"]
        for k in ("sseo", "ssen", "ssuo", "ssun", "ssvo", "ssvn", "dn", "dun", "dvn", "rru", "rrv", "taubx", "tauby",
                  "taub", "taus"):
            v3[k] = f2[k]
        ones2 = F2(np.ones(g.shape2()))
        v3.update(dt=np.float64(pd["dt"]), cnpar=np.float64(pd["cnpar"]), kmin=F2(np.ones(g.shape2())),
                  kumin=F2(np.ones(g.shape2())), kvmin=F2(np.ones(g.shape2())), ss=zero3(), nn=zero3(), zc=zero3(),
                  rad=f3["rad"], a=f2["a"], g1=f2["g1"], g2=f2["g2"], alpha=zero3(), beta=zero3(), rk=None,
                  avmback=np.float64(pd["avmback"]), avhback=np.float64(pd["avhback"]),
                  do_numerical_analyses=False, nummix3d_s=None, nummix2d_s=None, phymix3d_s=None,
                  phymix2d_s=None, nummix3d_t=None, nummix2d_t=None, phymix3d_t=None, phymix2d_t=None,
                  numdis3d=None, numdis2d=None, light=None, tke=f3["tke"], eps=f3["eps"])
        # kumin_pmz / kvmin_pmz (ip_blumberg_mellor_lin.F90:114,145): 1, the only value the reference
        # assigns them (adaptive_coordinates.F90:237-238)
        v3.update(kumin_pmz=F2(np.ones(g.shape2())), kvmin_pmz=F2(np.ones(g.shape2())))
        for k in ("kmin", "kumin", "kvmin", "kumin_pmz", "kvmin_pmz"):
            v3[k].a = v3[k].a.astype(np.int64)
        for v in (v2, v3):  # variables_2d/3d re-export the domain's index bounds (use domain)
            v.update(imin=g.imin, imax=g.imax, jmin=g.jmin, jmax=g.jmax, kmax=g.kmax)
        P.add_module_namespace("variables_2d", **v2)
        P.add_module_namespace("variables_3d", **v3)
        P.add_module_namespace("meteo", tausx=f2["tausx"], tausy=f2["tausy"], airp=f2["airp"], swr=f2["swr"],
                               shf=f2["shf"], albedo=zero2())
        # GOTM's turbulence module (un-vendored): gotm.F90's 1D column arrays under the local names
        # of its use-renames; PARABOLIC_VISCOSITY fills them itself and never calls do_turbulence
        col = lambda: fs.FArr(np.zeros(g.kmax + 1), [0])  # noqa: E731
        P.add_module_namespace("turbulence", tke1d=col(), eps1d=col(), l1d=col(), num1d=col(), nuh1d=col(),
                               cde=np.float64(0.5477), do_turbulence=self._no_turbulence)
        P.add_module_namespace("halo_zones", h_tag=10, hu_tag=11, hv_tag=12, d_tag=20, du_tag=21, dv_tag=22,
                               z_tag=30, u_tag=31, v_tag=32, update_2d_halo=lambda *a, **k: None,
                               update_3d_halo=lambda *a, **k: None, wait_halo=lambda *a, **k: None)
        timers = {f"tim_{n}": q for q, n in enumerate(
            "adv advh adv3d adv3dh salt temp mixanalysis bottfrict integr2d uvadv uvadvh uvdiff momentum momentumh "
            "sealevel sealevelh dpthupdate startmcr stopmcr bottfrict3d intpress uumomentum uumomentumh vvmomentum "
            "vvmomentumh coords wwmomentum wwmomentumh uvadv3d uvadv3dh uvdiff3d stresses3d stresses3dh tempH saltH "
            "eqstate slowbfrict slowterms integr3d check3df temph salth gotm gotmturb gotmh".split())}
        P.add_module_namespace("getm_timers", tic=lambda *a: None, toc=lambda *a: None, **timers)
        P.add_module_namespace("bdy_3d", do_bdy_3d=lambda *a, **k: None, init_bdy_3d=lambda *a, **k: None,
                               bdy3d_tmrlx=False, bdy3d_tmrlx_ucut=0.0, bdy3d_tmrlx_max=0.0, bdy3d_tmrlx_min=0.0)
        P.add_module_namespace("exceptions", getm_error=self._error)
        P.add_module_namespace("time", julianday=0, secondsofday=0, month=1, yearday=1)
        for f in FILES:
            P.load(f)
        # prescribed viscosity (CONSTANT_VISCOSITY): the turbulence interface is inert; with
        # PARABOLIC_VISCOSITY gotm.F90 runs its own profile. The shear/stratification inputs of the
        # closure (ss_nn) are never read by either
        if c.pi.get("viscosity", 0) == 1:
            P.load("src/3d/gotm.F90")
        else:
            P.procs["gotm"] = lambda *a, **k: None
        P.procs["ss_nn"] = lambda *a, **k: None
        P.procs["tke_eps_advect_3d"] = lambda *a, **k: None
        P.procs["do_residual"] = lambda *a, **k: None
        if c.bdy is None:
            P.procs["update_2d_bdy"] = lambda *a, **k: None
        P.procs["check_3d_fields"] = lambda *a, **k: None
        m2 = P.modules["m2d"]
        m2.dtm = np.float64(pd["dtm"])
        m2.mm = pi["MM"]
        m2.vel2d_adv_split, m2.vel2d_adv_hor = pi["vel2d_adv_split"], pi["vel2d_adv_hor"]
        m2.am, m2.an_method, m2.residual, m2.sealevel_check, m2.bdy2d_ramp = (np.float64(-1.0), 0, -1,
                                                                              int(pi.get("sealevel_check", 0)), -1)
        if c.bdy is not None:
            b, n = c.bdy, c.bdy.npoints()
            m2.bdy2d_ramp = b.ramp
            m2.bdyfmt_2d = 2  # NETCDF (cppdefs.h:88): data placed in bdy_data before each micro step
            m2.bdy_data = fs.FArr(np.zeros(n), [1])
            m2.bdy_data_u = fs.FArr(np.zeros(n) if b.data_u is None else b.data_u.copy(), [1])
            m2.bdy_data_v = fs.FArr(np.zeros(n) if b.data_v is None else b.data_v.copy(), [1])
        m3 = P.modules["m3d"]
        m3.m = pi["M"]
        m3.vel3d_adv_split, m3.vel3d_adv_hor, m3.vel3d_adv_ver = (pi["vel3d_adv_split"], pi["vel3d_adv_hor"],
                                                                  pi["vel3d_adv_ver"])
        m3.calc_temp, m3.calc_salt, m3.bdy3d, m3.advect_turbulence = True, True, False, False
        m3.ip_fac, m3.ip_ramp, m3.vel_check = np.float64(pd["ip_fac"]), -1, 0
        m3.vert_cord = 1
        tm = P.modules["temperature"]
        tm.temp_adv_split, tm.temp_adv_hor, tm.temp_adv_ver = (pi["temp_adv_split"], pi["temp_adv_hor"],
                                                               pi["temp_adv_ver"])
        tm.temp_ah, tm.temp_check, tm.ncid = np.float64(pd["temp_AH"]), 0, -1
        tm.swr_bot_refl_frac = np.float64(pd["swr_bot_refl_frac"])
        tm.swr_min_bot_frac = np.float64(pd["swr_min_bot_frac"])
        sm = P.modules["salinity"]
        sm.salt_adv_split, sm.salt_adv_hor, sm.salt_adv_ver = (pi["salt_adv_split"], pi["salt_adv_hor"],
                                                               pi["salt_adv_ver"])
        sm.salt_ah, sm.salt_check = np.float64(pd["salt_AH"]), 0
        eq = P.modules["eqstate"]
        eq.eqstate_method = int(pi.get("eqstate_method", 1))
        eq.t0, eq.s0, eq.dtr0, eq.dsr0 = (np.float64(pd["T0"]), np.float64(pd["S0"]), np.float64(pd["dtr0"]),
                                          np.float64(pd["dsr0"]))
        ipm = P.modules["internal_pressure"]
        ipm.ip_method = pi["ip_method"]
        ipm.zz = zero3()
        P.modules["advection"].init_advection()
        # sigma coordinates' first call sets the SAVEd equidistant switch and ga (coordinates.F90)
        P.procs["sigma_coordinates"](True)

    @staticmethod
    def _bdy_domain(b):
        """The domain module's boundary description (bdy_spec.F90:225-290) for an OpenBoundaries."""
        if b is None:
            return dict(openbdy=False, have_boundaries=False, nwb=0, nnb=0, neb=0, nsb=0)
        out = dict(openbdy=True, have_boundaries=True, nsbv=b.npoints())
        names = (("nwb", "wi", "wfj", "wlj"), ("nnb", "nj", "nfi", "nli"), ("neb", "ei", "efj", "elj"),
                 ("nsb", "sj", "sfi", "sli"))
        index, types, k = [], [], 1
        for side, (cnt, a, f, l) in zip(b.sides, names):
            out[cnt] = len(side)
            out[a] = fs.FArr(np.array([x[0] for x in side] or [0], np.int64), [1])
            out[f] = fs.FArr(np.array([x[1] for x in side] or [0], np.int64), [1])
            out[l] = fs.FArr(np.array([x[2] for x in side] or [0], np.int64), [1])
            for (_, first, last, typ) in side:
                index.append(k)
                types.append(typ)
                k += last - first + 1
        out["bdy_index"] = fs.FArr(np.array(index, np.int64), [1])
        out["bdy_2d_type"] = fs.FArr(np.array(types, np.int64), [1])
        return out

    @staticmethod
    def _no_turbulence(*a, **k):
        raise fs.FortranStop("do_turbulence: the GOTM closure is not part of this configuration")

    def _error(self, where, msg):
        raise fs.FortranStop(f"{where}: {msg}")

    def F2(self, a):
        g = self.g
        return fs.FArr(np.asfortranarray(np.asarray(a).T.copy()), [g.imin - 2, g.jmin - 2])

    def F3(self, a):
        g = self.g
        return fs.FArr(np.asfortranarray(np.transpose(np.asarray(a, np.float64), (2, 1, 0)).copy()),
                       [g.imin - 2, g.jmin - 2, 0])

    @staticmethod
    def N(fa):
        a = fa.a
        return np.ascontiguousarray(a.T if a.ndim == 2 else np.transpose(a, (2, 1, 0)))

    def time_loop(self, n0, count, runtype=4):
        tz = self.f2
        m2 = self.P.modules["m2d"]
        m3 = self.P.modules["m3d"]
        zeros = self.F2(np.zeros(self.g.shape2()))
        b = self.c.bdy
        for n in range(n0, n0 + count):
            if b is not None:  # the harness's boundary data of micro step n (the reference reads files)
                if b.amp is not None:
                    m2.bdy_data.a[:] = b.amp * np.sin(2.0 * np.pi * (n * m2.dtm) / b.period + b.phase)
                else:
                    m2.bdy_data.a[:] = b.data
            m2.integrate_2d(runtype, n, self.f2["tausx"], self.f2["tausy"], self.f2["airp"])
            if n % m3.m == 0:
                m3.integrate_3d(runtype, n)
        del tz, zeros

    def state(self):
        out = {}
        for k in S.F2_NAMES:
            out["f2_" + k] = self.N(self.f2[k.lower()])
        for k in S.F3_NAMES:
            out["f3_" + k] = self.N(self.f3[k.lower()])
        return out


def bdy_case():
    """12 x 10 x 4 shelf with a segment of each 2D boundary type on each side: CLAMPED (west),
    ZERO_GRADIENT (north), SOMMERFELD (east), FLATHER_ELEV (south); harmonic elevations (amplitude
    0.3 m, period 120 s = 8 micro steps, phase varying along the boundary), a ramp over 16 micro
    steps, and a constant bdy_data_v for the Flather segment."""
    g = S.Grid(12, 10, 4, 1000.0, 1000.0)
    b = S.OpenBoundaries(west=[(g.imin, g.jmin + 2, g.jmax - 2, S.CLAMPED)],
                         north=[(g.jmax, g.imin + 3, g.imax - 3, S.ZERO_GRADIENT)],
                         east=[(g.imax, g.jmin + 2, g.jmax - 2, S.SOMMERFELD)],
                         south=[(g.jmin, g.imin + 3, g.imax - 3, S.FLATHER_ELEV)], ramp=16, amp=0.3, period=120.0)
    b.phase = 0.1 * np.arange(b.npoints())
    b.data_v = np.full(b.npoints(), 0.02)
    return S.baroclinic_case(nx=12, ny=10, kmax=4, recipe="shelf", M=4, dt3=60.0, seed=3, bdy=b)


def ip_case(method):
    """12 x 10 x 5 islands basin (30% land) with another internal pressure method: 2
    (BLUMBERG_MELLOR_LIN, ip_blumberg_mellor_lin.F90), 3 (Z_INTERPOL, ip_z_interpol.F90), 7 (STELLING_VANKESTER,
    ip_stelling_vankester.F90), 4 (SONG_WRIGHT, ip_song_wright.F90) or 5
    (CHU_FAN, ip_chu_fan.F90). The stratified recipe on a varying bed, so that the height slopes
    and the vertical buoyancy gradients both enter the gradient."""
    c = S.baroclinic_case(nx=12, ny=10, kmax=5, recipe="islands", land=0.3, M=4, dt3=60.0, seed=7)
    c.pi["ip_method"] = method
    return c


def phys_case(eqstate_method, parabolic, reflection, seed=8):
    """12 x 10 x 5 islands basin (30% land) with the options of do_temperature, gotm and do_eqstate
    that the configurations leave off: short-wave radiation (swr 50-350 W/m2 and Jerlov type I
    attenuation A = 0.58, g1 = 0.35 m, g2 = 23 m, perturbed per column) and a surface heat flux of
    either sign, with the top layer of a few columns below the freezing point (the sea-ice clamp of
    the heat flux); optionally bottom reflection of the light (swr_bot_refl_frac = 0.2); the
    nonlinear equation of state (2: UNESCO80, 3: Jackett et al. 2006); optionally the
    PARABOLIC_VISCOSITY profile with background viscosity and diffusivity; the NaN sweep of the
    elevations every second micro step (warnings only)."""
    c = S.baroclinic_case(nx=12, ny=10, kmax=5, recipe="islands", land=0.3, M=4, dt3=60.0, seed=seed)
    rng = np.random.default_rng(seed + 100)
    g = c.grid
    wet = c.az >= 1
    c.pi.update(radiation=1, eqstate_method=eqstate_method, viscosity=1 if parabolic else 0, sealevel_check=-2)
    c.f2["swr"][...] = np.where(wet, rng.uniform(50.0, 350.0, g.shape2()), 0.0)
    c.f2["shf"][...] = np.where(wet, rng.uniform(-150.0, 100.0, g.shape2()), 0.0)
    c.f2["A"][...] = S.F32(0.58) + 0.02 * rng.uniform(-1, 1, g.shape2())
    c.f2["g1"][...] = S.F32(0.35) + 0.05 * rng.uniform(-1, 1, g.shape2())
    c.f2["g2"][...] = S.F32(23.0) + 2.0 * rng.uniform(-1, 1, g.shape2())
    T = c.f3["T"]
    cold = wet & (rng.uniform(size=g.shape2()) < 0.25)
    T[g.kmax][cold] = -2.5  # below -0.0575*S for S >= 30
    if reflection:
        c.pd["swr_bot_refl_frac"] = 0.2
    if parabolic:
        c.pd.update(avmback=1e-5, avhback=2e-6)
        c.f2["taub"][...] = np.where(wet, rng.uniform(0.0, 2e-4, g.shape2()), 0.0)
    S._eqstate(c)  # initial density and buoyancy of the modified temperature (linear)
    return c


def write(c, name):
    out = {"meta": np.array([c.grid.nx, c.grid.ny, c.grid.kmax, c.grid.dx, c.grid.dy])}
    r = RefBc(c)
    # the inputs are the state the reference starts from: its first sigma_coordinates call (in
    # RefBc) recomputes the layer heights from H and the elevations, which may differ from the
    # case's in the last bit
    for k, v in r.state().items():
        out["in_" + k] = np.array(v, copy=True)  # state() views the arrays the run then updates
    for k, v in zip(("az", "au", "av", "ax"), c.masks()):
        out["in_" + k] = v
    out["in_pd"] = np.array([c.pd[n] for n in S.PD_NAMES])
    out["in_pi"] = np.array([c.pi[n] for n in S.PI_NAMES])
    out["names_pd"] = np.array(S.PD_NAMES)
    out["names_pi"] = np.array(S.PI_NAMES)
    if c.bdy is not None:
        b = c.bdy
        out["bdy_counts"] = np.array([len(x) for x in b.sides])
        out["bdy_seg"] = np.array([[p_, f, l, t] for (p_, f, l, t) in b.segments()])
        out["bdy_ramp"] = np.array(b.ramp)
        out["bdy_amp"], out["bdy_phase"], out["bdy_period"] = b.amp, b.phase, np.array(b.period)
        out["bdy_data_v"] = b.data_v
    # two macro steps (M = 4 micro steps each)
    r.time_loop(1, 8)
    for k, v in r.state().items():
        out["out_" + k] = v
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


def nan_check_fixture():
    """tests/golden/reference_sealevel_nan.npz: the reference's sealevel_nan_check
    (sealevel.F90:172-314) on elevation fields holding NaN, +-Inf, HUGE, subnormal and ordinary
    values, in the interior and in the halo, with land points among them. For each field: the number
    of interior points that sealevel_nandum classifies as not below HUGE (recorded from the
    reference's own per-point calls), the last such point in loop order, and whether sealevel(loop)
    stops (getm_error) with sealevel_check = 1 and with sealevel_check = -1."""
    c = S.baroclinic_case(nx=9, ny=7, kmax=3, recipe="islands", land=0.3, M=4, dt3=60.0, seed=5)
    g = c.grid
    rng = np.random.default_rng(21)
    fields = []
    z0 = c.f2["z"].copy()
    fields.append(z0.copy())  # clean
    z = z0.copy()
    pts = [(g.jmin + 1, g.imin + 2, np.nan), (g.jmin + 3, g.imin, np.inf), (g.jmax, g.imax, np.finfo(np.float64).max),
           (g.jmin, g.imax - 1, -np.inf), (g.jmin + 2, g.imin + 4, 5e-324), (g.jmin - 1, g.imin + 1, np.nan)]
    for (j, i, v) in pts:
        z[j - (g.jmin - 2), i - (g.imin - 2)] = v
    fields.append(z)
    z = z0.copy()
    z[rng.uniform(size=z.shape) < 0.2] = np.nan  # random NaNs, halo included
    fields.append(z)
    out = {"meta": np.array([g.nx, g.ny, g.kmax, g.dx, g.dy]), "in_az": c.az}
    for q, zf in enumerate(fields):
        res = {}
        for chk in (1, -1):
            cc = c.copy()
            cc.f2["z"][...] = zf
            cc.pi["sealevel_check"] = chk
            r = RefBc(cc)
            calls = []
            orig = r.P.procs["sealevel_nandum"]

            def spy(a, b, idum, _orig=orig, _calls=calls):
                ret = _orig(a, b, idum)
                _calls.append(int(ret[2]) if ret else 2)
                return ret

            r.P.procs["sealevel_nandum"] = spy
            r.P.modules["m2d"].dtm = np.float64(0.0)  # the sweep sees the field as given
            stopped = False
            try:
                r.P.procs["sealevel"](1)
            except fs.FortranStop:
                stopped = True
            res[chk] = (stopped, calls[2:])  # the first two calls are the compiler self-test
        flags = np.array(res[1][1])
        out[f"z{q}"] = zf
        out[f"count{q}"] = np.array(int((flags == 2).sum()))
        ii, jj = np.meshgrid(np.arange(g.imin, g.imax + 1), np.arange(g.jmin, g.jmax + 1))
        hit = np.flatnonzero(flags == 2)
        out[f"last{q}"] = np.array([ii.ravel()[hit[-1]], jj.ravel()[hit[-1]]] if hit.size else [0, 0])
        out[f"stops{q}"] = np.array([res[1][0], res[-1][0]])
    path = os.path.join(HERE, "reference_sealevel_nan.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}")


RESTART_2D = ["z", "zo", "U", "SlUx", "Slru", "V", "SlVx", "Slrv", "ssen", "ssun", "ssvn", "sseo", "ssuo", "ssvo",
              "Uinto", "Vinto"]
RESTART_3D = ["uu", "vv", "ww", "uuEx", "vvEx", "tke", "eps", "num", "nuh", "hn", "T", "S"]


def hotstart_fixture():
    """tests/golden/reference_hotstart.npz: the reference's hotstart re-initialisation. A state is run
    8 micro steps by the reference; the interiors of its restart fields (write_restart_ncdf.F90:86-204,
    runtype 4) are the 'file'. A fresh state of the same basin gets those interiors (the halos keep
    the fresh state's values, as read_restart_ncdf leaves them), with a non-zero U and V placed on a
    closed velocity point, then the reference's postinit_2d and postinit_3d (m2d.F90:325-403,
    m3d.F90:302-412) run with hotstart = .true.: out_* is the state after them."""
    c = S.baroclinic_case(nx=12, ny=10, kmax=5, recipe="islands", land=0.3, M=4, dt3=60.0, seed=7)
    r = RefBc(c.copy())
    r.time_loop(1, 8)
    done = r.state()
    g = c.grid
    it = (slice(2, 2 + g.ny), slice(2, 2 + g.nx))
    out = {"meta": np.array([g.nx, g.ny, g.kmax, g.dx, g.dy])}
    fresh = c.copy()
    file2 = {k: done["f2_" + k][it].copy() for k in RESTART_2D}
    file3 = {k: done["f3_" + k][(slice(None),) + it].copy() for k in RESTART_3D}
    # a closed U point and a closed V point of the interior with a non-zero value in the file
    ju, iu = [int(x) for x in np.argwhere(c.au[it] == 0)[0]]
    jv, iv = [int(x) for x in np.argwhere(c.av[it] == 0)[0]]
    file2["U"][ju, iu] = 0.125
    file2["V"][jv, iv] = -0.25
    file2["Uinto"][ju, iu] = 3.0
    for k, v in file2.items():
        fresh.f2[k][it] = v
        out["file_f2_" + k] = v
    for k, v in file3.items():
        fresh.f3[k][(slice(None),) + it] = v
        out["file_f3_" + k] = v
    pre = c.copy()  # the state before the file is read (the case's initial state)
    for k in S.F2_NAMES:
        out["in_f2_" + k] = pre.f2[k]
    for k in S.F3_NAMES:
        out["in_f3_" + k] = pre.f3[k]
    for k, v in zip(("az", "au", "av", "ax"), c.masks()):
        out["in_" + k] = v
    out["in_pd"] = np.array([c.pd[n] for n in S.PD_NAMES])
    out["in_pi"] = np.array([c.pi[n] for n in S.PI_NAMES])
    out["names_pd"] = np.array(S.PD_NAMES)
    out["names_pi"] = np.array(S.PI_NAMES)
    rh = RefBc(fresh)
    rh.P.modules["m2d"].postinit_2d(4, np.float64(c.pd["dtm"]), True)
    rh.P.modules["m3d"].postinit_3d(4, np.float64(c.pd["dt"]), True)
    for k, v in rh.state().items():
        out["out_" + k] = v
    path = os.path.join(HERE, "reference_hotstart.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


def main():
    which = sys.argv[1:] or ["closed", "bdy", "ip2", "ip3", "ip4", "ip5", "ip6", "ip7", "phys3", "phys2", "nan", "hotstart"]
    if "closed" in which:
        write(S.baroclinic_case(nx=12, ny=10, kmax=4, recipe="shelf", M=4, dt3=60.0, seed=3),
              "reference_mode_split.npz")
    if "bdy" in which:
        write(bdy_case(), "reference_mode_split_bdy.npz")
    for m in (2, 3, 4, 5, 6, 7):
        if f"ip{m}" in which:
            write(ip_case(m), f"reference_mode_split_ip{m}.npz")
    if "phys3" in which:  # Jackett 2006, PARABOLIC_VISCOSITY, radiation with bottom reflection
        write(phys_case(3, parabolic=True, reflection=True), "reference_mode_split_phys3.npz")
    if "nan" in which:
        nan_check_fixture()
    if "hotstart" in which:
        hotstart_fixture()
    if "phys2" in which:  # UNESCO80, prescribed viscosity, radiation without reflection
        write(phys_case(2, parabolic=False, reflection=False, seed=9), "reference_mode_split_phys2.npz")


if __name__ == "__main__":
    main()
