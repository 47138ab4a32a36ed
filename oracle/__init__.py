"""CPU oracle -- TEST INFRASTRUCTURE ONLY.

ctypes bindings for ``oracle/_build/liboracle.so``, the C++ restatement of GETM's hot-path
routines (``getm_oracle.hpp``). Imported only by ``tests/``, by the smoke check in
``__graft_entry__.py`` and by ``bench.py``'s CPU-baseline leg, always as the checker or the
reported CPU baseline -- never as the measured or shipped path.

Arrays are numpy arrays in the reference layout: a 3D field of the haloed index space
``(imin-2:imax+2, jmin-2:jmax+2, 0:kmax)`` is a C-contiguous ``(kmax+1, nj, ni)`` array (which is
the Fortran column-major layout), a 2D field is ``(nj, ni)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_NATIVE_PATH = os.path.join(_HERE, "_build", "liboracle_native.so")
_lib = None
BUILD_FLAGS = {"portable": "g++ -O3 -march=x86-64-v2 -fopenmp -ffp-contract=off",
               "native": "g++ -O3 -march=native -fopenmp -ffp-contract=off"}
variant = "portable"  # which build lib() loads


class OrDom(C.Structure):
    _fields_ = [
        ("imin", C.c_int), ("imax", C.c_int), ("jmin", C.c_int), ("jmax", C.c_int), ("kmax", C.c_int),
        ("sj", C.c_longlong), ("sk", C.c_longlong),
        ("dx", C.c_double), ("dy", C.c_double), ("ard1", C.c_double),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP, no FP contraction)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


def use_native_build() -> bool:
    """Build (with the machine's own g++) and select the -march=native oracle for timing on this
    host's cores; returns False, keeping the portable build, if that build fails. Call before the
    first oracle routine runs."""
    global variant
    if _lib is not None:
        return variant == "native"
    try:
        # always rebuilt (-B): a library tuned for another machine's CPU must not be reused
        subprocess.check_call(["make", "-s", "-B", "-C", _HERE, "native"], stdout=subprocess.DEVNULL,
                              stderr=subprocess.DEVNULL)
    except (OSError, subprocess.CalledProcessError):
        return False
    variant = "native"
    return True


def lib():
    global _lib
    if _lib is None:
        path = _NATIVE_PATH if variant == "native" else _LIB_PATH
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
        _declare(_lib)
    return _lib


P = C.c_void_p


def _declare(L):
    for suf, R in (("d", C.c_double), ("f", C.c_float)):
        getattr(L, f"or_adv_split_u_{suf}").argtypes = [P, R, P, P, P, P, P, P, R, C.c_int, R, P, P]
        getattr(L, f"or_adv_split_v_{suf}").argtypes = [P, R, P, P, P, P, P, P, R, C.c_int, R, P, P]
        fw = getattr(L, f"or_adv_split_w_{suf}")
        fw.argtypes = [P, R, P, P, P, P, P, R, C.c_int, C.c_int, P, C.c_int]
        fw.restype = C.c_longlong
        f3 = getattr(L, f"or_do_advection_3d_{suf}")
        f3.argtypes = [P, P, P, P, P, R, P, P, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, R, C.c_int,
                       P, P, C.c_int]
        f3.restype = C.c_longlong
        f2 = getattr(L, f"or_do_advection_{suf}")
        f2.argtypes = [P, P, P, P, P, R, P, P, P, P, P, P, P, C.c_int, C.c_int, R, C.c_int, P, P]
        f2.restype = C.c_int
        getattr(L, f"or_tridiagonal_{suf}").argtypes = [C.c_int, C.c_int, C.c_int, P, P, P, P, P]
        getattr(L, f"or_tracer_vdiff_{suf}").argtypes = [P, R, R, R, P, P, P, P, P]
        tc = getattr(L, f"or_tracer_content_{suf}")
        tc.argtypes = [P, P, P, P]
        tc.restype = C.c_double
        ts = getattr(L, f"or_tracer_steps_{suf}")
        ts.argtypes = [P, P, P, P, P, C.c_int, R, P, P, P, P, P, P, P, P, P, C.c_int, C.c_int,
                       C.c_int, R, R, R, C.c_int]
        ts.restype = C.c_longlong
        rc = getattr(L, f"or_recon_{suf}")
        rc.argtypes = [C.c_int, P, P, P, P, P, C.c_longlong]
        rc.restype = C.c_int
    L.or_tracer_steps_tl.argtypes = [P, P, P, P, P, C.c_int, C.c_double, P, P, P, P, P, P, P, P, P, P, P,
                                     C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
    L.or_tracer_steps_tl.restype = C.c_longlong
    L.or_derive_uvx.argtypes = [P, P, P, P, P]
    L.or_build_masks.argtypes = [P, P, P, P, P, P]
    for suf in ("d", "f"):
        fn = getattr(L, f"or_bc_steps_{suf}")
        fn.argtypes = [P, P, C.c_int, C.c_int]
        fn.restype = C.c_longlong
        fn = getattr(L, f"or_bc_call_{suf}")
        fn.argtypes = [P, P, C.c_int, C.c_int]
        fn.restype = C.c_int
    L.or_bc_sizes.argtypes = [P]
    L.or_sealevel_nan_check.argtypes = [P, P, P, P]
    L.or_sealevel_nan_check.restype = C.c_longlong


# routine ids of or_bc_call (oracle_capi.cpp)
BC_ROUTINES = ["bottom_friction", "uv_advect_2d", "umomentum", "vmomentum", "sealevel", "depth_update",
               "start_macro", "bottom_friction_3d", "internal_pressure", "uu_momentum_3d", "vv_momentum_3d",
               "sigma_coordinates", "ww_momentum_3d", "uv_advect_3d", "stresses_3d", "do_eqstate",
               "slow_bottom_friction", "slow_terms", "integrate_2d", "integrate_3d", "gotm_parabolic", "sw_radiation",
               "update_2d_bdy", "hotstart_postinit"]


def bc_sizes():
    out = (C.c_int * 4)()
    lib().or_bc_sizes(out)
    return tuple(out)


def bc_steps(case, n0: int, count: int):
    """time_loop over micro steps n0..n0+count-1 on a code_b200.state.BcCase (in place)."""
    from code_b200.state import oracle_struct, read_back_ipar

    s = oracle_struct(case)
    dom = OrDom(case.grid.imin, case.grid.imax, case.grid.jmin, case.grid.jmax, case.grid.kmax, case.grid.ni,
                case.grid.ni * case.grid.nj, case.grid.dx, case.grid.dy, case.grid.ard1)
    fn = lib().or_bc_steps_d if case.dtype3 == np.float64 else lib().or_bc_steps_f
    r = fn(C.addressof(dom), C.addressof(s), n0, count)
    read_back_ipar(case, s)
    if r < 0:
        raise ValueError("bc_steps failed")


def bc_call(case, routine: str, arg: int = 0):
    """One routine of the mode-split step on a BcCase (in place)."""
    from code_b200.state import oracle_struct, read_back_ipar

    s = oracle_struct(case)
    dom = OrDom(case.grid.imin, case.grid.imax, case.grid.jmin, case.grid.jmax, case.grid.kmax, case.grid.ni,
                case.grid.ni * case.grid.nj, case.grid.dx, case.grid.dy, case.grid.ard1)
    fn = lib().or_bc_call_d if case.dtype3 == np.float64 else lib().or_bc_call_f
    r = fn(C.addressof(dom), C.addressof(s), BC_ROUTINES.index(routine), arg)
    read_back_ipar(case, s)
    if r != 0:
        raise ValueError(f"{routine} failed ({r})")


def sealevel_nan_check(grid, z):
    """sealevel_nan_check (sealevel.F90:172-314): (count, i, j) of the interior elevations that are
    not below HUGE; (i, j) is the last such point in the reference's loop order (None if none)."""
    dom = OrDom(grid.imin, grid.imax, grid.jmin, grid.jmax, grid.kmax, grid.ni, grid.ni * grid.nj, grid.dx, grid.dy,
                grid.ard1)
    i, j = C.c_int(0), C.c_int(0)
    n = lib().or_sealevel_nan_check(C.addressof(dom), _p(np.ascontiguousarray(z, np.float64)), C.byref(i), C.byref(j))
    return int(n), (int(i.value), int(j.value)) if n > 0 else None


def _p(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous, "oracle arrays must be C-contiguous numpy"
    return a.ctypes.data


def _suf(dtype) -> str:
    if dtype == np.float64:
        return "d"
    if dtype == np.float32:
        return "f"
    raise TypeError(f"unsupported dtype {dtype}")


class Grid:
    """Index space of one run: interior imin..imax x jmin..jmax, levels 0..kmax, halo 2."""

    def __init__(self, nx: int, ny: int, kmax: int, dx: float, dy: float, imin: int = 1, jmin: int = 1):
        self.nx, self.ny, self.kmax = nx, ny, kmax
        self.imin, self.jmin = imin, jmin
        self.imax, self.jmax = imin + nx - 1, jmin + ny - 1
        self.ni, self.nj, self.nk = nx + 4, ny + 4, kmax + 1
        self.dx, self.dy = float(dx), float(dy)
        self.ard1 = 1.0 / (self.dx * self.dy)  # domain.F90:596

    def dom(self) -> OrDom:
        return OrDom(self.imin, self.imax, self.jmin, self.jmax, self.kmax, self.ni, self.ni * self.nj,
                     self.dx, self.dy, self.ard1)

    def shape3(self):
        return (self.nk, self.nj, self.ni)

    def shape2(self):
        return (self.nj, self.ni)


class Oracle:
    """Reference-named wrappers around the C++ restatement for one Grid."""

    def __init__(self, grid):
        # any object with the Grid attributes (imin..kmax, ni, nj, dx, dy, ard1)
        self.g = grid
        self._dom = OrDom(grid.imin, grid.imax, grid.jmin, grid.jmax, grid.kmax, grid.ni, grid.ni * grid.nj,
                          grid.dx, grid.dy, grid.ard1)
        self._pd = C.addressof(self._dom)
        self.L = lib()

    # --- masks -----------------------------------------------------------------------------
    def derive_uvx(self, az):
        g = self.g
        au = np.zeros(g.shape2(), np.int32)
        av = np.zeros(g.shape2(), np.int32)
        ax = np.zeros(g.shape2(), np.int32)
        self.L.or_derive_uvx(self._pd, _p(az), _p(au), _p(av), _p(ax))
        return au, av, ax

    def build_masks(self, az, au, av, ax):
        g = self.g
        out = np.zeros((8,) + g.shape2(), np.uint8)
        self.L.or_build_masks(self._pd, _p(az), _p(au), _p(av), _p(ax), _p(out))
        names = ["updateH", "uflux", "vflux", "xflux", "uupdateU", "vupdateV", "uflux_U", "vflux_V"]
        return {n: out[q] for q, n in enumerate(names)}

    # --- routines --------------------------------------------------------------------------
    def recon(self, scheme, cfl, fuu, fu, fd):
        s = _suf(cfl.dtype)
        out = np.empty_like(cfl)
        getattr(self.L, f"or_recon_{s}")(scheme, _p(cfl), _p(fuu), _p(fu), _p(fd), _p(out), cfl.size)
        return out

    def adv_split_u(self, dt, f, fi, Di, adv, U, DU, splitfac, scheme, AH, mask_flux, mask_update):
        s = _suf(f.dtype)
        getattr(self.L, f"or_adv_split_u_{s}")(self._pd, dt, _p(f), _p(fi), _p(Di), _p(adv), _p(U), _p(DU),
                                              splitfac, scheme, AH, _p(mask_flux), _p(mask_update))

    def adv_split_v(self, dt, f, fi, Di, adv, V, DV, splitfac, scheme, AH, mask_flux, mask_update):
        s = _suf(f.dtype)
        getattr(self.L, f"or_adv_split_v_{s}")(self._pd, dt, _p(f), _p(fi), _p(Di), _p(adv), _p(V), _p(DV),
                                              splitfac, scheme, AH, _p(mask_flux), _p(mask_update))

    def adv_split_w(self, dt, f, fi, hi, adv, ww, splitfac, scheme, tag, az, itersmax):
        s = _suf(f.dtype)
        return getattr(self.L, f"or_adv_split_w_{s}")(self._pd, dt, _p(f), _p(fi), _p(hi), _p(adv), _p(ww),
                                                     splitfac, scheme, tag, _p(az), itersmax)

    def do_advection_3d(self, masks, dt, f, uu, vv, ww, hu, hv, ho, hn, split, hscheme, vscheme, AH, tag,
                        hires=None, advres=None, adv_ver_iterations=1):
        az, au, av, ax = masks
        s = _suf(f.dtype)
        r = getattr(self.L, f"or_do_advection_3d_{s}")(
            self._pd, _p(az), _p(au), _p(av), _p(ax), dt, _p(f), _p(uu), _p(vv), _p(ww), _p(hu), _p(hv),
            _p(ho), _p(hn), split, hscheme, vscheme, AH, tag, _p(hires), _p(advres), adv_ver_iterations)
        if r < 0:
            raise ValueError("do_advection_3d: invalid split/scheme")
        return r

    def do_advection(self, masks, dt, f, U, V, DU, DV, Do, Dn, split, scheme, AH, tag, Dires=None, advres=None):
        az, au, av, ax = masks
        s = _suf(f.dtype)
        r = getattr(self.L, f"or_do_advection_{s}")(
            self._pd, _p(az), _p(au), _p(av), _p(ax), dt, _p(f), _p(U), _p(V), _p(DU), _p(DV), _p(Do), _p(Dn),
            split, scheme, AH, tag, _p(Dires), _p(advres))
        if r < 0:
            raise ValueError("do_advection: invalid split/scheme")

    def tridiagonal(self, kmax, fi, lt, au, bu, cu, du):
        s = _suf(au.dtype)
        value = np.zeros_like(au)
        getattr(self.L, f"or_tridiagonal_{s}")(kmax, fi, lt, _p(au), _p(bu), _p(cu), _p(du), _p(value))
        return value

    def tracer_vdiff(self, dt, cnpar, avmol, S, hn, nuh, az, src=None):
        s = _suf(S.dtype)
        getattr(self.L, f"or_tracer_vdiff_{s}")(self._pd, dt, cnpar, avmol, _p(S), _p(hn), _p(nuh), _p(az),
                                               _p(src))

    def tracer_content(self, f, h, az):
        return getattr(self.L, f"or_tracer_content_{_suf(f.dtype)}")(self._pd, _p(f), _p(h), _p(az))

    def tracer_steps(self, masks, nsteps, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme,
                     AH, cnpar, avmol, adv_ver_iterations=1):
        az, au, av, ax = masks
        s = _suf(f.dtype)
        r = getattr(self.L, f"or_tracer_steps_{s}")(
            self._pd, _p(az), _p(au), _p(av), _p(ax), nsteps, dt, _p(f), _p(uu), _p(vv), _p(ww), _p(hu), _p(hv),
            _p(ho), _p(hn), _p(nuh), split, hscheme, vscheme, AH, cnpar, avmol, adv_ver_iterations)
        if r < 0:
            raise ValueError("tracer_steps: invalid split/scheme")
        return r

    def tracer_steps_tl(self, masks, nsteps, dt, f, df, uu, vv, ww, hu, hv, ho, hn, nuh, dnuh, split, hscheme,
                        vscheme, AH, cnpar, avmol):
        """Tangent-linear FP64 tracer steps (dual numbers, getm_tangent.hpp): f and df advance in
        place; df is the derivative of the state in the direction (df, dnuh) of (initial tracer, nuh)."""
        az, au, av, ax = masks
        r = self.L.or_tracer_steps_tl(
            self._pd, _p(az), _p(au), _p(av), _p(ax), nsteps, dt, _p(f), _p(df), _p(uu), _p(vv), _p(ww), _p(hu),
            _p(hv), _p(ho), _p(hn), _p(nuh), None if dnuh is None else _p(dnuh), split, hscheme, vscheme, AH, cnpar,
            avmol)
        if r < 0:
            raise ValueError("tracer_steps_tl: invalid split/scheme")
        return r
