"""Generates tests/golden/*.npz: inputs and outputs of the reference's OWN Fortran routines.

Runs here, where the reference is mounted (GETM_REFERENCE, default /root/reference), through
fortran_subset.py (the reference's .F90 files preprocessed with cpp and executed in IEEE double
precision). The fixtures then pin both the C++ oracle (tests/test_golden_cpu.py) and the CUDA
kernels (tests/test_gpu_golden.py) to the reference's results, cell by cell.

    python tests/golden/make_golden.py

Routines executed (file:line in the reference):
  getm_tridiagonal                 src/futils/tridiagonal.F90:8-51
  adv_interfacial_reconstruction   src/2d/advection.F90:785-879
  init_advection (masks)           src/2d/advection.F90:204-354
  adv_split_u / adv_split_v        src/2d/adv_split_u.F90, src/2d/adv_split_v.F90
  adv_split_w (incl. iterations)   src/3d/adv_split_w.F90
  do_advection_3d (all splits)     src/3d/advection_3d.F90:120-598
  do_salinity (advection + implicit vertical diffusion)   src/3d/salinity.F90:225-435
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

import fortran_subset as fs  # noqa: E402
from code_b200 import cases  # noqa: E402

NAMES3 = ("f", "uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")


class RefRun:
    """The reference's routines loaded for one grid (module state set from a Case)."""

    def __init__(self, c):
        self.c = c
        g = self.g = c.grid
        P = self.P = fs.Program()
        P.add_module_namespace("domain", imin=g.imin, imax=g.imax, jmin=g.jmin, jmax=g.jmax, kmax=g.kmax,
                               dx=g.dx, dy=g.dy, ard1=g.ard1, ioff=0, joff=0, az=self.F2(c["az"]),
                               au=self.F2(c["au"]), av=self.F2(c["av"]), ax=self.F2(c["ax"]),
                               h=self.F2(np.zeros(g.shape2())))
        P.add_module_namespace("halo_zones", h_tag=10, hu_tag=11, hv_tag=12, d_tag=20, du_tag=21, dv_tag=22,
                               z_tag=30, u_tag=31, v_tag=32, update_2d_halo=lambda *a, **k: None,
                               update_3d_halo=lambda *a, **k: None, wait_halo=lambda *a, **k: None)
        P.add_module_namespace("getm_timers", tic=lambda *a: None, toc=lambda *a: None,
                               **{n: q for q, n in enumerate(["tim_adv", "tim_advh", "tim_adv3d", "tim_adv3dh",
                                                              "tim_salt", "tim_mixanalysis", "tim_temp"])})
        P.add_module_namespace("parameters", g=np.float64(np.float32(9.81)), rho_0=np.float64(1025.0),
                               avmols=np.float64(np.float32(1.1e-9)), avmolt=np.float64(np.float32(1.4e-7)))
        for f in ("src/futils/tridiagonal.F90", "src/2d/advection.F90", "src/2d/adv_split_u.F90",
                  "src/2d/adv_split_v.F90", "src/3d/advection_3d.F90", "src/3d/adv_split_w.F90"):
            P.load(f)
        P.modules["advection"].init_advection()

    # layout conversion: product arrays are C-order (k, j, i); Fortran arrays are (i, j, k)
    def F2(self, a):
        g = self.g
        return fs.FArr(np.asfortranarray(np.asarray(a).T.copy()), [g.imin - 2, g.jmin - 2])

    def F3(self, a):
        g = self.g
        return fs.FArr(np.asfortranarray(np.transpose(np.asarray(a), (2, 1, 0)).copy()), [g.imin - 2, g.jmin - 2, 0])

    @staticmethod
    def N(fa):
        a = fa.a
        return np.ascontiguousarray(a.T if a.ndim == 2 else np.transpose(a, (2, 1, 0)))

    def do_advection_3d(self, dt, split, hs, vs, AH, tag, iters=1):
        c = self.c
        self.P.modules["advection_3d"].adv_ver_iterations = iters
        f = self.F3(c["f"])
        hires, advres = self.F3(np.zeros_like(c["f"])), self.F3(np.zeros_like(c["f"]))
        args = [self.F3(c[n]) for n in ("uu", "vv", "ww", "hun", "hvn", "ho", "hn")]
        self.P.modules["advection_3d"].do_advection_3d(dt, f, *args, split, hs, vs, AH, tag, hires, advres)
        self.P.modules["advection_3d"].adv_ver_iterations = 1
        return self.N(f), self.N(hires), self.N(advres)

    def do_salinity(self, nsteps, dt, cnpar, split, hs, vs, AH):
        """do_salinity(n) for n = 1..nsteps with the module state of variables_3d / salinity."""
        c, g = self.c, self.g
        P = self.P
        S = self.F3(c["f"])
        v3 = dict(dt=np.float64(dt), cnpar=np.float64(cnpar), hn=self.F3(c["hn"]), ho=self.F3(c["ho"]),
                  nuh=self.F3(c["nuh"]), uu=self.F3(c["uu"]), vv=self.F3(c["vv"]), ww=self.F3(c["ww"]),
                  hun=self.F3(c["hun"]), hvn=self.F3(c["hvn"]), s=S, rk=None, kmin=self.F2(np.zeros(g.shape2())),
                  do_numerical_analyses=False, nummix3d_s=None, nummix2d_s=None, phymix3d_s=None,
                  phymix2d_s=None)
        P.add_module_namespace("variables_3d", **v3)
        P.add_module_namespace("variables_2d", fwf_int=self.F2(np.zeros(g.shape2())))
        if "salinity" not in P.modules or not hasattr(P.modules["salinity"], "do_salinity"):
            P.load("src/3d/salinity.F90")
        ns = P.modules["salinity"]
        ns.salt_adv_split, ns.salt_adv_hor, ns.salt_adv_ver = split, hs, vs
        ns.salt_ah = np.float64(AH)
        ns.salt_check = 0
        for n in range(1, nsteps + 1):
            ns.do_salinity(n)
        return self.N(P.modules["variables_3d"].s)


def main():
    out = {}
    # routine-level: tridiagonal and the limiter library on random inputs
    rng = np.random.default_rng(2024)
    P = fs.Program().load("src/futils/tridiagonal.F90")
    kmax = 9
    tri = {k: rng.uniform(-1, 0, (kmax + 1,)) for k in ("au", "cu")}
    tri["bu"] = 2.5 + rng.uniform(0, 1, kmax + 1)
    tri["du"] = rng.normal(size=kmax + 1)
    for fi, lt in ((1, 9), (0, 9), (2, 5)):
        val = fs.FArr(np.zeros(kmax + 1, order="F"), [0])
        P.procs["getm_tridiagonal"](kmax, fi, lt, *[fs.FArr(np.asfortranarray(tri[k].copy()), [0])
                                                    for k in ("au", "bu", "cu", "du")], val)
        out[f"tri_{fi}_{lt}"] = val.a.copy()
    for k, v in tri.items():
        out[f"tri_in_{k}"] = v

    c = cases.random_case(nx=10, ny=8, kmax=4, seed=7)
    rr = RefRun(c)
    adv = rr.P.modules["advection"]
    n = 4000
    rec_in = {"cfl": rng.uniform(0, 1, n), "fuu": rng.normal(size=n), "fu": rng.normal(size=n),
              "fd": rng.normal(size=n)}
    # include exact ties and zero slopes
    rec_in["fd"][:200] = rec_in["fu"][:200]
    rec_in["fuu"][200:400] = rec_in["fu"][200:400]
    rec_in["cfl"][400:450] = 0.0
    for k, v in rec_in.items():
        out[f"rec_in_{k}"] = v
    for scheme in (1, 3, 4, 5, 6):
        out[f"rec_{scheme}"] = np.array([adv.adv_interfacial_reconstruction(scheme, rec_in["cfl"][q], rec_in["fuu"][q],
                                                                            rec_in["fu"][q], rec_in["fd"][q])
                                         for q in range(n)], dtype=np.float64)

    for k in ("az", "au", "av", "ax"):
        out[f"case_{k}"] = c[k]
    for k in NAMES3:
        out[f"case_{k}"] = c[k]
    out["case_meta"] = np.array([c.grid.nx, c.grid.ny, c.grid.kmax, c.grid.dx, c.grid.dy, c.par["dt"]])
    for nm, arr in (("updateH", adv.mask_updateh), ("uflux", adv.mask_uflux), ("vflux", adv.mask_vflux),
                    ("xflux", adv.mask_xflux), ("uupdateU", adv.mask_uupdateu), ("vupdateV", adv.mask_vupdatev)):
        out[f"mask_{nm}"] = rr.N(arr).astype(np.uint8)
    dt = c.par["dt"]
    configs = []
    for split in (0, 1, 2, 3):
        for hs, vs in ((4, 4), (6, 6), (1, 5), (3, 1), (5, 0), (0, 6)):
            for tag in (10, 31, 32):
                if vs == 0 and split == 3:
                    continue
                AH = 3.0 if hs == 5 else 0.0
                f, h, a = rr.do_advection_3d(dt, split, hs, vs, AH, tag)
                key = f"adv3d_{split}_{hs}_{vs}_{tag}"
                out[key + "_f"], out[key + "_h"], out[key + "_a"] = f, h, a
                configs.append((split, hs, vs, tag, AH))
    out["adv3d_configs"] = np.array(configs, dtype=np.float64)
    # vertical sub-iterations: w-Courant numbers up to ~3 (adv_ver_iterations = 2 and 4)
    cw = cases.random_case(nx=10, ny=8, kmax=4, seed=7)
    cw["ww"] = cw["ww"] * 6.0
    rw = RefRun(cw)
    for iters in (2, 4):
        fs.WRITES.writes = 0
        f, h, a = rw.do_advection_3d(dt, 2, 6, 6, 0.0, 10, iters)
        out[f"adv3d_iter{iters}_f"], out[f"adv3d_iter{iters}_h"], out[f"adv3d_iter{iters}_a"] = f, h, a
        # each column over the cap prints two lines (adv_split_w.F90:225-226)
        out[f"adv3d_iter{iters}_warn"] = np.array([fs.WRITES.writes // 2])
    out["case_ww6"] = cw["ww"]
    # do_salinity: advection + implicit vertical diffusion, 3 steps, reference default cnpar=0.9
    # (a single-precision literal) and cnpar=1
    for cn_name, cn in (("09", float(np.float32(0.9))), ("10", 1.0)):
        rs = RefRun(c)
        out[f"salt_{cn_name}"] = rs.do_salinity(3, dt, cn, 2, 6, 6, 0.0)
    path = os.path.join(HERE, "reference_hot_path.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB, {len(out)} arrays)")


if __name__ == "__main__":
    main()
