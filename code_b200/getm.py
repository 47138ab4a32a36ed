"""Host-side mirror of GETM's hot-path routines over the CUDA library's C ABI.

Each method keeps the reference subroutine's name, argument order and argument meaning
(``do_advection_3d(dt,f,uu,vv,ww,hu,hv,ho,hn,split,hscheme,vscheme,AH,tag,hires,advres)``,
advection_3d.F90:120-122, and so on) and operates on CUDA tensors laid out like the reference's
arrays (see :mod:`code_b200.grid`). torch supplies device memory and the stream only; all
arithmetic runs in the library's kernels. There is no CPU fallback: without the compiled library
or a CUDA device every call raises.

Errors: where the reference stops (``stop 'do_advection_3d: tag is invalid'``) the library
returns a status code and this layer raises :class:`GetmError` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from .grid import Grid

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libgetm_b200.so")

# scheme / split / tag ids (advection.F90:55-62, halo_zones.F90:25-27, advection_3d.F90:42)
NOSPLIT, FULLSPLIT, HALFSPLIT, HVSPLIT = 0, 1, 2, 3
NOADV, UPSTREAM, UPSTREAM_2DH, P2, SUPERBEE, MUSCL, P2_PDM, J7, FCT, P2_2DH = range(10)
H_TAG, D_TAG, U_TAG, V_TAG, W_TAG = 10, 20, 31, 32, 33

ERRORS = {-1: "GETM_ERR_ARG", -2: "GETM_ERR_CUDA", -3: "GETM_ERR_UNSUPPORTED", -4: "GETM_ERR_CHECK",
          -5: "GETM_ERR_TIMEOUT", -6: "GETM_ERR_NOMEM", -7: "GETM_ERR_STATE",
          -8: "GETM_ERR_TOO_LARGE"}


class GetmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()
P = C.c_void_p
I = C.c_int
D = C.c_double
F = C.c_float


class AdvGrid(C.Structure):
    _fields_ = [("mask_uflux", P), ("mask_vflux", P), ("mask_uupdate", P), ("mask_vupdate", P),
                ("mask_finalise", P), ("az", P)]


# name -> argtypes (restype int unless listed in _RESTYPES)
_PROTOS = {
    "getm_ctx_create": [P, P, P],
    "getm_ctx_destroy": [P],
    "getm_ctx_set_stream": [P, P],
    "getm_ctx_take_warnings": [P, P],
    "getm_ctx_last_error": [P],
    "getm_version": [],
    "getm_init_advection": [P, P, P, P, P],
    "getm_adv_grid_for_tag": [P, I, P],
    "getm_adv_split_u": [P, I, D, P, P, P, P, P, P, D, I, D, P, P],
    "getm_adv_split_v": [P, I, D, P, P, P, P, P, P, D, I, D, P, P],
    "getm_adv_split_w": [P, D, P, P, P, P, P, D, I, I, P, I],
    "getm_adv_split_u_f32": [P, I, F, P, P, P, P, P, P, F, I, F, P, P],
    "getm_adv_split_v_f32": [P, I, F, P, P, P, P, P, P, F, I, F, P, P],
    "getm_adv_split_w_f32": [P, F, P, P, P, P, P, F, I, I, P, I],
    "getm_do_advection_3d": [P, D, P, P, P, P, P, P, P, P, I, I, I, D, I, P, P, I],
    "getm_do_advection_3d_f32": [P, F, P, P, P, P, P, P, P, P, I, I, I, F, I, P, P, I],
    "getm_tridiagonal_columns": [P, I, I, I, I, P, P, P, P, P],
    "getm_tracer_vdiff": [P, D, D, D, P, P, P, P, P],
    "getm_tracer_vdiff_f32": [P, F, F, F, P, P, P, P, P],
    "getm_tracer_vdiff_noalloc": [P, P, D, D, D, P, P, P, P, P],
    "getm_set_open_boundaries": [P, P],
    "getm_set_bdy_data": [P, P, P, P],
    "getm_tracer_step_record": [P, D, P, P, P, P, P, P, P, P, P, I, I, I, D, D, D, P, P],
    "getm_tracer_step_record_f32": [P, F, P, P, P, P, P, P, P, P, P, I, I, I, F, F, F, P, P],
    "getm_tracer_step_adjoint": [P, D, P, P, P, P, P, P, P, P, P, P, I, I, I, D, D, D, P, P],
    "getm_tracer_step_adjoint_f32": [P, F, P, P, P, P, P, P, P, P, P, P, I, I, I, F, F, F, P, P],
    "getm_tracer_gradient": [P, I, I, D, P, P, P, P, P, P, P, P, P, I, I, I, D, D, D, P, P, P, P],
    "getm_tracer_gradient_f32": [P, I, I, F, P, P, P, P, P, P, P, P, P, I, I, I, F, F, F, P, P, P, P],
    "getm_tracer_step": [P, D, P, P, P, P, P, P, P, P, P, I, I, I, D, D, D, I],
    "getm_tracer_step_f32": [P, F, P, P, P, P, P, P, P, P, P, I, I, I, F, F, F, I],
    "getm_tracer_content": [P, P, P, P, P],
    "getm_tracer_content_f32": [P, P, P, P, P],
    "getm_check_3d_fields": [P, P, P, D, D, P],
    "getm_set_vector_sweeps": [I],
    "getm_set_fused_micro_step": [I],
    "getm_set_fp32_micro_steps": [I],
    "getm_timers_enable": [P, I],
    "getm_timers_reset": [P],
    "getm_timers_read": [P, I, P, P],
    "getm_timer_name": [I],
    "getm_integrate_2d": [P, P, I],
    "getm_integrate_3d": [P, P, I],
    "getm_time_loop": [P, P, I, I],
    "getm_bottom_friction": [P, P, I],
    "getm_uv_advect": [P, P],
    "getm_momentum": [P, P, I],
    "getm_umomentum": [P, P],
    "getm_vmomentum": [P, P],
    "getm_update_2d_bdy": [P, P, I],
    "getm_sealevel": [P, P, I],
    "getm_depth_update": [P, P],
    "getm_internal_pressure": [P, P],
    "getm_do_eqstate": [P, P],
    "getm_gotm": [P, P],
    "getm_sw_radiation": [P, P],
    "getm_sealevel_nan_check": [P, P, P, P, P],
    "getm_halo_pack": [P, P, I, I, I, I, P],
    "getm_restart_fields": [I, P, P, P, P],
    "getm_restart_write": [P, P, I, P, P],
    "getm_restart_read": [P, P, I, P, P],
    "getm_halo_unpack": [P, P, I, I, I, I, P],
}
_RESTYPES = {"getm_ctx_last_error": C.c_char_p, "getm_version": C.c_char_p, "getm_timer_name": C.c_char_p}
NTIMERS = 16


def lib():
    """Load the compiled library (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"CUDA library not built: {LIB_PATH} is missing "
                                   "(run __graft_entry__.build() or python code_b200/build.py)")
            L = C.CDLL(LIB_PATH)
            for name, args in _PROTOS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = _RESTYPES.get(name, C.c_int)
            _lib = L
    return _lib


def restart_fields(runtype: int):
    """State-table indices (f2, f3) of the restart file's fields for a runtype, in the file's order."""
    n2, n3 = C.c_int32(), C.c_int32()
    a = (C.c_int32 * 64)()
    b = (C.c_int32 * 64)()
    rc = lib().getm_restart_fields(runtype, a, C.byref(n2), b, C.byref(n3))
    if rc:
        raise GetmError(rc, "restart_fields")
    return list(a[:n2.value]), list(b[:n3.value])


def set_fp32_micro_steps(on: bool) -> bool:
    """Process-wide choice for the mixed step's micro steps: FP32 working copies of the 2D fields
    (the default) or the FP64 state arrays; returns the previous setting."""
    return bool(lib().getm_set_fp32_micro_steps(1 if on else 0))


def set_fused_micro_step(on: bool) -> bool:
    """Process-wide choice of the micro-step launches (sealevel + depth_update as one launch with
    the elevation ping-pong, bottom friction inside the mixed step's momentum advection; or the
    separate launches); returns the previous setting."""
    return bool(lib().getm_set_fused_micro_step(1 if on else 0))


def set_vector_sweeps(on: bool) -> bool:
    """Process-wide choice of the horizontal sweep kernels (vectorised where the layout allows, or
    the shared-memory tile sweeps everywhere); returns the previous setting."""
    return bool(lib().getm_set_vector_sweeps(1 if on else 0))


def exported_symbols():
    return list(_PROTOS)


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def _same_dtype(ref, *ts):
    for t in ts:
        if t is not None and t.dtype != ref.dtype:
            raise TypeError(f"dtype mismatch: {t.dtype} vs {ref.dtype}")


class Context:
    """One device context (getm_ctx): grid, stream, advection masks and scratch."""

    def __init__(self, grid: Grid, stream=None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("a CUDA device is required (no CPU fallback)")
        self.grid = grid
        self.L = lib()
        self._dom = grid.domain()
        if stream is None:
            stream = torch.cuda.current_stream()
        self.stream = stream
        h = P()
        self._check(self.L.getm_ctx_create(C.byref(self._dom), P(stream.cuda_stream), C.byref(h)), None)
        self.h = h

    # ------------------------------------------------------------------------------------------
    def _check(self, rc: int, h=0):
        if rc != 0:
            hh = self.h if h == 0 else h
            msg = self.L.getm_ctx_last_error(hh).decode() if hh else "context creation failed"
            raise GetmError(rc, msg)

    def close(self):
        if getattr(self, "h", None):
            self.L.getm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        self.stream = stream
        self._check(self.L.getm_ctx_set_stream(self.h, P(stream.cuda_stream)))

    def take_warnings(self) -> int:
        n = C.c_int64()
        self._check(self.L.getm_ctx_take_warnings(self.h, C.byref(n)))
        return n.value

    # ------------------------------------------------------------------------------------------
    def timers(self, enable: bool | None = None, reset: bool = False) -> dict:
        """Per-stage device timers (tic/toc of getm_timers): {name: (total_ms, launches)}."""
        if enable is not None:
            self._check(self.L.getm_timers_enable(self.h, 1 if enable else 0))
        out = {}
        for t in range(NTIMERS):
            ms, n = C.c_double(), C.c_int64()
            self._check(self.L.getm_timers_read(self.h, t, C.byref(ms), C.byref(n)))
            if n.value:
                out[self.L.getm_timer_name(t).decode()] = (ms.value, n.value)
        if reset:
            self._check(self.L.getm_timers_reset(self.h))
        return out

    def init_advection(self, az, au, av, ax):
        """init_advection (advection.F90:204-354) from int32 device masks."""
        self._masks = (az, au, av, ax)  # keep alive
        self._check(self.L.getm_init_advection(self.h, _ptr(az), _ptr(au), _ptr(av), _ptr(ax)))

    def adv_grid(self, tag: int) -> AdvGrid:
        g = AdvGrid()
        self._check(self.L.getm_adv_grid_for_tag(self.h, tag, C.byref(g)))
        return g

    def adv_split_u(self, dt, f, fi, Di, adv, U, DU, splitfac, scheme, AH, mask_flux, mask_update, nk=None):
        _same_dtype(f, fi, Di, adv, U, DU)
        nk = nk if nk is not None else (f.shape[0] if f.dim() == 3 else 1)
        fn = self.L.getm_adv_split_u if _is64(f) else self.L.getm_adv_split_u_f32
        self._check(fn(self.h, nk, dt, _ptr(f), _ptr(fi), _ptr(Di), _ptr(adv), _ptr(U), _ptr(DU), splitfac, scheme, AH,
                       _mask(mask_flux), _mask(mask_update)))

    def adv_split_v(self, dt, f, fi, Di, adv, V, DV, splitfac, scheme, AH, mask_flux, mask_update, nk=None):
        _same_dtype(f, fi, Di, adv, V, DV)
        nk = nk if nk is not None else (f.shape[0] if f.dim() == 3 else 1)
        fn = self.L.getm_adv_split_v if _is64(f) else self.L.getm_adv_split_v_f32
        self._check(fn(self.h, nk, dt, _ptr(f), _ptr(fi), _ptr(Di), _ptr(adv), _ptr(V), _ptr(DV), splitfac, scheme, AH,
                       _mask(mask_flux), _mask(mask_update)))

    def adv_split_w(self, dt, f, fi, hi, adv, ww, splitfac, scheme, tag, az, itersmax=1):
        _same_dtype(f, fi, hi, adv, ww)
        fn = self.L.getm_adv_split_w if _is64(f) else self.L.getm_adv_split_w_f32
        self._check(fn(self.h, dt, _ptr(f), _ptr(fi), _ptr(hi), _ptr(adv), _ptr(ww), splitfac, scheme, tag, _ptr(az),
                       itersmax))

    def do_advection_3d(self, dt, f, uu, vv, ww, hu, hv, ho, hn, split, hscheme, vscheme, AH, tag,
                        hires=None, advres=None, adv_ver_iterations=1):
        """do_advection_3d (advection_3d.F90:120-598); f is advanced in place."""
        _same_dtype(f, uu, vv, ww, hu, hv, ho, hn, hires, advres)
        fn = self.L.getm_do_advection_3d if _is64(f) else self.L.getm_do_advection_3d_f32
        self._check(fn(self.h, dt, _ptr(f), _ptr(uu), _ptr(vv), _ptr(ww), _ptr(hu), _ptr(hv), _ptr(ho), _ptr(hn),
                       split, hscheme, vscheme, AH, tag, _ptr(hires), _ptr(advres), adv_ver_iterations))

    def tridiagonal(self, kmax, fi, lt, au, bu, cu, du, value):
        """getm_tridiagonal (tridiagonal.F90:8-51) on the columns of [k][col] tensors."""
        ncol = au.shape[1]
        _need64(au, bu, cu, du, value)
        self._check(self.L.getm_tridiagonal_columns(self.h, ncol, kmax, fi, lt, _ptr(au), _ptr(bu), _ptr(cu),
                                                    _ptr(du), _ptr(value)))

    def tracer_vdiff(self, dt, cnpar, avmol, S, hn, nuh, az, src=None):
        """Vertical-diffusion solve of do_salinity / do_temperature (salinity.F90:348-389)."""
        _same_dtype(S, hn, nuh, src)
        fn = self.L.getm_tracer_vdiff if _is64(S) else self.L.getm_tracer_vdiff_f32
        self._check(fn(self.h, dt, cnpar, avmol, _ptr(S), _ptr(hn), _ptr(nuh), _ptr(az), _ptr(src)))

    def tracer_step(self, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH, cnpar, avmol,
                    adv_ver_iterations=1):
        """Advection + vertical diffusion of one tracer (the body of do_salinity)."""
        _same_dtype(f, uu, vv, ww, hu, hv, ho, hn, nuh)
        fn = self.L.getm_tracer_step if _is64(f) else self.L.getm_tracer_step_f32
        self._check(fn(self.h, dt, _ptr(f), _ptr(uu), _ptr(vv), _ptr(ww), _ptr(hu), _ptr(hv), _ptr(ho), _ptr(hn),
                       _ptr(nuh), split, hscheme, vscheme, AH, cnpar, avmol, adv_ver_iterations))

    # ---- open boundaries ---------------------------------------------------------------------
    def set_open_boundaries(self, bdy):
        """Open-boundary segments and elevation data (a code_b200.state.OpenBoundaries), used by
        integrate_2d / integrate_3d / time_loop from now on (None: closed domain)."""
        from .state import OpenBoundaries

        b = bdy if bdy is not None else OpenBoundaries()
        st = b.struct()
        self._check(self.L.getm_set_open_boundaries(self.h, C.byref(st)))

    def set_bdy_data(self, data, data_u=None, data_v=None):
        """New boundary elevations (and Flather velocities) per boundary point, numpy FP64."""
        import numpy as np

        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (data, data_u, data_v)]
        self._check(self.L.getm_set_bdy_data(self.h, *[None if a is None else a.ctypes.data for a in arrs]))

    # ---- adjoint of the tracer step --------------------------------------------------------
    def tape(self, dtype):
        """Allocates the tape of one step: (codes uint8[5*n3], g of the field's dtype)."""
        import torch

        n3 = self.grid.ni * self.grid.nj * (self.grid.kmax + 1)
        return (torch.empty(5 * n3, dtype=torch.uint8, device="cuda"),
                torch.empty(self.grid.shape3(), dtype=dtype, device="cuda"))

    def tracer_step_record(self, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH, cnpar,
                           avmol, tape):
        """getm_tracer_step that also writes the adjoint tape (see Context.tape)."""
        _same_dtype(f, uu, vv, ww, hu, hv, ho, hn, nuh, tape[1])
        fn = self.L.getm_tracer_step_record if _is64(f) else self.L.getm_tracer_step_record_f32
        self._check(fn(self.h, dt, _ptr(f), _ptr(uu), _ptr(vv), _ptr(ww), _ptr(hu), _ptr(hv), _ptr(ho), _ptr(hn),
                       _ptr(nuh), split, hscheme, vscheme, AH, cnpar, avmol, _ptr(tape[0]), _ptr(tape[1])))

    def tracer_step_adjoint(self, dt, fbar, nubar, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH,
                            cnpar, avmol, tape):
        """Adjoint of one recorded tracer step: fbar in place, nubar accumulated."""
        _same_dtype(fbar, nubar, uu, vv, ww, hu, hv, ho, hn, nuh, tape[1])
        fn = self.L.getm_tracer_step_adjoint if _is64(fbar) else self.L.getm_tracer_step_adjoint_f32
        self._check(fn(self.h, dt, _ptr(fbar), _ptr(nubar), _ptr(uu), _ptr(vv), _ptr(ww), _ptr(hu), _ptr(hv),
                       _ptr(ho), _ptr(hn), _ptr(nuh), split, hscheme, vscheme, AH, cnpar, avmol, _ptr(tape[0]),
                       _ptr(tape[1])))

    def tracer_gradient(self, nsteps, every, dt, f, uu, vv, ww, hu, hv, ho, hn, nuh, split, hscheme, vscheme, AH,
                        cnpar, avmol, fbar, nubar):
        """Checkpointed gradient over nsteps steps; returns (ms_forward, ms_reverse)."""
        _same_dtype(f, uu, vv, ww, hu, hv, ho, hn, nuh, fbar, nubar)
        fn = self.L.getm_tracer_gradient if _is64(f) else self.L.getm_tracer_gradient_f32
        a, r = C.c_float(), C.c_float()
        self._check(fn(self.h, nsteps, every, dt, _ptr(f), _ptr(uu), _ptr(vv), _ptr(ww), _ptr(hu), _ptr(hv),
                       _ptr(ho), _ptr(hn), _ptr(nuh), split, hscheme, vscheme, AH, cnpar, avmol, _ptr(fbar),
                       _ptr(nubar), C.byref(a), C.byref(r)))
        return a.value, r.value

    def tracer_content(self, f, h, az) -> float:
        out = C.c_double()
        fn = self.L.getm_tracer_content if _is64(f) else self.L.getm_tracer_content_f32
        self._check(fn(self.h, _ptr(f), _ptr(h), _ptr(az), C.byref(out)))
        return out.value

    # ---- mode-split step ----------------------------------------------------------------------
    def integrate_2d(self, st: "BcDevice", loop: int):
        """integrate_2d (m2d.F90:412-490) on a device state."""
        self._check(self.L.getm_integrate_2d(self.h, C.byref(st.c), loop))

    def integrate_3d(self, st: "BcDevice", n: int):
        """integrate_3d (m3d.F90:422-636) on a device state."""
        self._check(self.L.getm_integrate_3d(self.h, C.byref(st.c), n))

    def time_loop(self, st: "BcDevice", n0: int, count: int):
        """Micro steps n0..n0+count-1 of time_loop (integration.F90:98-172)."""
        self._check(self.L.getm_time_loop(self.h, C.byref(st.c), n0, count))

    # the substeps of integrate_2d / integrate_3d, one by one (reference routine names)
    def bottom_friction(self, st: "BcDevice", runtype: int):
        """bottom_friction (bottom_friction.F90:8-250)."""
        self._check(self.L.getm_bottom_friction(self.h, C.byref(st.c), runtype))

    def uv_advect(self, st: "BcDevice"):
        """uv_advect(U, V, DU, DV) (uv_advect.F90:8-310): UEx, VEx."""
        self._check(self.L.getm_uv_advect(self.h, C.byref(st.c)))

    def momentum(self, st: "BcDevice", n: int):
        """momentum (momentum.F90:8-60): umomentum and vmomentum in alternating order."""
        self._check(self.L.getm_momentum(self.h, C.byref(st.c), n))

    def umomentum(self, st: "BcDevice"):
        """umomentum (momentum.F90:69-223)."""
        self._check(self.L.getm_umomentum(self.h, C.byref(st.c)))

    def vmomentum(self, st: "BcDevice"):
        """vmomentum (momentum.F90:232-386)."""
        self._check(self.L.getm_vmomentum(self.h, C.byref(st.c)))

    def update_2d_bdy(self, st: "BcDevice", loop: int):
        """update_2d_bdy (update_2d_bdy.F90:8-186) with the context's open boundaries."""
        self._check(self.L.getm_update_2d_bdy(self.h, C.byref(st.c), loop))

    def sealevel(self, st: "BcDevice", loop: int):
        """sealevel (sealevel.F90:8-163), with its NaN sweep when sealevel_check asks for one."""
        self._check(self.L.getm_sealevel(self.h, C.byref(st.c), loop))

    def depth_update(self, st: "BcDevice"):
        """depth_update (depth_update.F90:8-148)."""
        self._check(self.L.getm_depth_update(self.h, C.byref(st.c)))

    def internal_pressure(self, st: "BcDevice"):
        """do_internal_pressure (internal_pressure.F90:181-274) with the state's ip_method."""
        self._check(self.L.getm_internal_pressure(self.h, C.byref(st.c)))

    def do_eqstate(self, st: "BcDevice"):
        """do_eqstate (eqstate.F90:94-261) with the state's eqstate_method."""
        self._check(self.L.getm_do_eqstate(self.h, C.byref(st.c)))

    def gotm(self, st: "BcDevice"):
        """gotm (gotm.F90:96-163) with PARABOLIC_VISCOSITY (viscosity = 1; no-op otherwise)."""
        self._check(self.L.getm_gotm(self.h, C.byref(st.c)))

    def sw_radiation(self, st: "BcDevice"):
        """The short-wave radiation profile rad of do_temperature (temperature.F90:452-465)."""
        self._check(self.L.getm_sw_radiation(self.h, C.byref(st.c)))

    def sealevel_nan_check(self, z):
        """sealevel_nan_check (sealevel.F90:172-314): (count, (i, j) of the last finding or None)."""
        n, i, j = C.c_int64(), C.c_int32(), C.c_int32()
        _need64(z)
        self._check(self.L.getm_sealevel_nan_check(self.h, _ptr(z), C.byref(n), C.byref(i), C.byref(j)))
        return int(n.value), ((int(i.value), int(j.value)) if n.value else None)

    # hotstart: the restart file's fields (write_restart_ncdf.F90 / read_restart_ncdf.F90)
    def restart_write(self, st: "BcDevice", runtype: int) -> dict:
        """The restart fields' interiors as FP64 numpy arrays {name: (nk, ny, nx) or (ny, nx)}."""
        import numpy as np

        from . import state as S

        i2, i3 = restart_fields(runtype)
        g = self.grid
        h2 = [np.zeros((g.ny, g.nx)) for _ in i2]
        h3 = [np.zeros((g.kmax + 1, g.ny, g.nx)) for _ in i3]
        p2 = (C.c_void_p * max(1, len(h2)))(*[a.ctypes.data for a in h2])
        p3 = (C.c_void_p * max(1, len(h3)))(*[a.ctypes.data for a in h3])
        self._check(self.L.getm_restart_write(self.h, C.byref(st.c), runtype, p2, p3 if h3 else None))
        out = {S.F2_NAMES[q]: a for q, a in zip(i2, h2)}
        out.update({S.F3_NAMES[q]: a for q, a in zip(i3, h3)})
        return out

    def restart_read(self, st: "BcDevice", runtype: int, fields: dict):
        """Hotstart from restart-field interiors {name: FP64 array} (see restart_write)."""
        import numpy as np

        from . import state as S

        i2, i3 = restart_fields(runtype)
        h2 = [np.ascontiguousarray(fields[S.F2_NAMES[q]], np.float64) for q in i2]
        h3 = [np.ascontiguousarray(fields[S.F3_NAMES[q]], np.float64) for q in i3]
        p2 = (C.c_void_p * max(1, len(h2)))(*[a.ctypes.data for a in h2])
        p3 = (C.c_void_p * max(1, len(h3)))(*[a.ctypes.data for a in h3])
        self._check(self.L.getm_restart_read(self.h, C.byref(st.c), runtype, p2, p3 if h3 else None))

    # halo rows of a slab decomposition (update_3d_halo / update_2d_halo of the parallel build)
    def halo_pack(self, f, j_first: int, nrows: int, buf):
        """Rows j_first..j_first+nrows-1 of every level of f (3D, or 2D) into the packed buffer buf."""
        nk = f.shape[0] if f.dim() == 3 else 1
        self._check(self.L.getm_halo_pack(self.h, _ptr(f), f.element_size(), nk, j_first, nrows, _ptr(buf)))

    def halo_unpack(self, f, j_first: int, nrows: int, buf):
        """The packed buffer buf into rows j_first..j_first+nrows-1 of every level of f."""
        nk = f.shape[0] if f.dim() == 3 else 1
        self._check(self.L.getm_halo_unpack(self.h, _ptr(f), f.element_size(), nk, j_first, nrows, _ptr(buf)))

    def check_3d_fields(self, f, az, minval, maxval) -> int:
        _need64(f)
        st = C.c_int64()
        self._check(self.L.getm_check_3d_fields(self.h, _ptr(f), _ptr(az), minval, maxval, C.byref(st)))
        return st.value


def _need64(*ts):
    """The FP64-only entry points take FP64 tensors only (the library reads them as double)."""
    import torch

    for t in ts:
        if t is not None and t.dtype != torch.float64:
            raise TypeError(f"expected float64, got {t.dtype}")


def _is64(t) -> bool:
    import torch

    if t.dtype == torch.float64:
        return True
    if t.dtype == torch.float32:
        return False
    raise TypeError(f"unsupported dtype {t.dtype}")


def _mask(m):
    if m is None:
        return None
    if isinstance(m, int):
        return m
    return _ptr(m)


class BcState(C.Structure):
    """Mirror of getm_bc_state (include/getm_b200.h)."""

    _fields_ = [("f2", P * 59), ("f3", P * 24), ("az", P), ("au", P), ("av", P), ("ax", P), ("par", D * 23),
                ("ipar", C.c_int32 * 25), ("prec3d", C.c_int32)]


class BcDevice:
    """Device copy of a mode-split state (code_b200.state.BcCase) plus its C table."""

    def __init__(self, case=None, dtype3=None, tensors=None, pd=None, pi=None, compensated=True):
        """compensated: with FP32 3D fields, keep the compensated storage of T and S (Tlo, Slo)."""
        import torch

        from . import state as S

        if tensors is None:
            dt3 = dtype3 or (torch.float64 if case.dtype3 == "float64" else torch.float32)
            t = {}
            for n in S.F2_NAMES:
                t["f2_" + n] = torch.from_numpy(case.f2[n]).cuda()
            for n in S.F3_NAMES:
                if n in ("Tlo", "Slo"):
                    # FP16, scaled carried errors, starting at zero
                    if dt3 == torch.float32 and compensated:
                        t["f3_" + n] = torch.zeros(case.f3[n].shape, dtype=torch.float16, device="cuda")
                    continue
                t["f3_" + n] = torch.from_numpy(case.f3[n]).to(dt3).cuda()
            for n, m in zip(("az", "au", "av", "ax"), case.masks()):
                t[n] = torch.from_numpy(m).cuda()
            pd, pi = dict(case.pd), dict(case.pi)
        self.t = tensors if tensors is not None else t
        self.pd, self.pi = pd, pi
        f3dt = self.t["f3_uu"].dtype
        self.prec = 8 if f3dt == torch.float64 else 4
        c = BcState()
        # optional fields (S.OPTIONAL_F2 / OPTIONAL_F3) that a state does not hold cross as NULL
        for q, n in enumerate(S.F2_NAMES):
            t2 = self.t.get("f2_" + n)
            assert t2 is not None or n in S.OPTIONAL_F2, n
            c.f2[q] = None if t2 is None else _ptr(t2)
        for q, n in enumerate(S.F3_NAMES):
            t3 = self.t.get("f3_" + n)
            assert t3 is not None or n in S.OPTIONAL_F3, n
            assert t3 is None or t3.dtype == (torch.float16 if n in ("Tlo", "Slo") else f3dt)
            c.f3[q] = None if t3 is None else _ptr(t3)
        c.az, c.au, c.av, c.ax = (_ptr(self.t[n]) for n in ("az", "au", "av", "ax"))
        for q, n in enumerate(S.PD_NAMES):
            c.par[q] = float(pd[n])
        for q, n in enumerate(S.PI_NAMES):
            c.ipar[q] = int(pi[n])
        c.prec3d = self.prec
        self.c = c

    def masks(self):
        return tuple(self.t[n] for n in ("az", "au", "av", "ax"))

    def ipar(self) -> dict:
        from . import state as S

        return {n: int(self.c.ipar[q]) for q, n in enumerate(S.PI_NAMES)}

    def to_host(self, case):
        """Copy the device fields back into a BcCase (3D fields cast to the case's dtype)."""
        from . import state as S

        for n in S.F2_NAMES:
            if "f2_" + n in self.t:
                case.f2[n][...] = self.t["f2_" + n].cpu().numpy()
        for n in S.F3_NAMES:
            if "f3_" + n in self.t:
                case.f3[n][...] = self.t["f3_" + n].cpu().numpy().astype(case.dtype3)
        for q, n in enumerate(S.PI_NAMES):
            case.pi[n] = int(self.c.ipar[q])
        return case
