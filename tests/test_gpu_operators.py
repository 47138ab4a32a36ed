"""The substeps of the mode-split step called one by one through the C ABI (getm_bottom_friction,
getm_uv_advect, getm_momentum / umomentum / vmomentum, getm_update_2d_bdy, getm_sealevel,
getm_depth_update, getm_internal_pressure, getm_do_eqstate, getm_gotm, getm_sw_radiation,
getm_sealevel_nan_check), each against the oracle's routine of the same name on the same state;
and the options of the step that the configurations leave off (short-wave radiation and surface
heat flux, PARABOLIC_VISCOSITY, the UNESCO80 and Jackett 2006 equations of state, the NaN sweep
of the elevations) through getm_time_loop against the reference's executed fixtures and the
oracle.

Tolerance (FP64): bit for bit where the routine has no transcendental function; 1e-12 of the
field's largest magnitude where the device's log or exp enters (bottom friction, radiation), whose
last bit may differ from the host C library's."""
import numpy as np
import pytest

import oracle
from code_b200 import state as S
from code_b200.getm import BcDevice, GetmError
from helpers import make_ctx
from test_golden_bc_cpu import GOLD_NAN, GOLD_PHYS, gold_names, load_case

pytestmark = pytest.mark.gpu


def field_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.nanmax(np.abs(b))), 1e-300)
    return float(np.nanmax(np.abs(a - b))) / scale


def started_case(recipe="islands", bdy=False, steps=10, **kw):
    """A state a few micro steps into a run (the oracle's time loop), so that every field is
    populated and moving."""
    if bdy:
        g = S.Grid(30, 24, 6, 1000.0, 1000.0)
        b = S.OpenBoundaries(west=[(g.imin, g.jmin + 2, g.jmax - 2, S.CLAMPED)],
                             north=[(g.jmax, g.imin + 3, g.imax - 3, S.ZERO_GRADIENT)],
                             east=[(g.imax, g.jmin + 2, g.jmax - 2, S.SOMMERFELD)],
                             south=[(g.jmin, g.imin + 3, g.imax - 3, S.FLATHER_ELEV)], ramp=8, amp=0.3,
                             period=300.0)
        c = S.baroclinic_case(nx=30, ny=24, kmax=6, recipe="shelf", M=5, seed=2, bdy=b)
    else:
        c = S.baroclinic_case(nx=40, ny=28, kmax=10, recipe=recipe, M=5, dt3=60.0, seed=11, land=0.3, **kw)
    oracle.bc_steps(c, 1, steps)
    return c


def gpu_call(c, method, *args):
    import torch

    ctx, _ = make_ctx(c)
    if c.bdy is not None:
        ctx.set_open_boundaries(c.bdy)
    st = BcDevice(c)
    getattr(ctx, method)(st, *args)
    torch.cuda.synchronize()
    out = st.to_host(c.copy())
    return out


ROUTINES_2D = [("bottom_friction", "bottom_friction", (4,), 4, 1e-12), ("uv_advect", "uv_advect_2d", (), 0, 0.0),
               ("umomentum", "umomentum", (), 0, 0.0), ("vmomentum", "vmomentum", (), 0, 0.0),
               ("sealevel", "sealevel", (11,), 0, 0.0), ("depth_update", "depth_update", (), 0, 0.0)]


@pytest.mark.parametrize("bdy", [False, True], ids=["closed", "open boundaries"])
@pytest.mark.parametrize("method,ref,args,arg,tol", ROUTINES_2D, ids=[r[0] for r in ROUTINES_2D])
def test_2d_substep_vs_oracle(method, ref, args, arg, tol, bdy):
    c = started_case(bdy=bdy)
    want = c.copy()
    oracle.bc_call(want, ref, arg)
    got = gpu_call(c, method, *args)
    for k in S.F2_NAMES:
        e = field_err(got.f2[k], want.f2[k])
        assert e <= tol, (k, e)


def test_momentum_alternates_like_reference():
    """getm_momentum runs umomentum then vmomentum when ufirst2d is set and the other order
    otherwise, toggling the switch (momentum.F90:44-52)."""
    import torch

    for first in (0, 1):
        c = started_case()
        c.pi["ufirst2d"] = first
        want = c.copy()
        if first:
            oracle.bc_call(want, "umomentum")
            oracle.bc_call(want, "vmomentum")
        else:
            oracle.bc_call(want, "vmomentum")
            oracle.bc_call(want, "umomentum")
        ctx, _ = make_ctx(c)
        st = BcDevice(c)
        ctx.momentum(st, 11)
        torch.cuda.synchronize()
        got = st.to_host(c.copy())
        assert got.pi["ufirst2d"] == 1 - first
        for k in S.F2_NAMES:
            assert np.array_equal(got.f2[k], want.f2[k], equal_nan=True), k


def test_update_2d_bdy_vs_oracle():
    """update_2d_bdy at micro step 11 (harmonic elevations, ramp over 8 steps, all four types)."""
    c = started_case(bdy=True)
    want = c.copy()
    oracle.bc_call(want, "update_2d_bdy", 11)
    got = gpu_call(c, "update_2d_bdy", 11)
    assert not np.array_equal(want.f2["z"], c.f2["z"])  # the boundary moved
    for k in S.F2_NAMES:
        assert np.array_equal(got.f2[k], want.f2[k], equal_nan=True), k


@pytest.mark.parametrize("method", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("prec", [8, 4], ids=["fp64", "fp32"])
def test_internal_pressure_vs_oracle(method, prec):
    """getm_internal_pressure = do_internal_pressure with the state's ip_method: FP64 bit for bit;
    the FP32 state within 1e-5 of the FP64 oracle's gradients (relative to their largest value)."""
    import torch

    c = started_case()
    c.pi["ip_method"] = method
    want = c.copy()
    oracle.bc_call(want, "internal_pressure")
    cc = c if prec == 8 else c.copy(dtype3=np.float32)
    ctx, _ = make_ctx(cc)
    st = BcDevice(cc, dtype3=torch.float64 if prec == 8 else torch.float32)
    ctx.internal_pressure(st)
    torch.cuda.synchronize()
    got = st.to_host(cc.copy())
    for k in ("idpdx", "idpdy"):
        if prec == 8:
            assert np.array_equal(got.f3[k], want.f3[k]), k
        else:
            assert field_err(got.f3[k], want.f3[k]) < 1e-5, k


@pytest.mark.parametrize("method", [1, 2, 3])
def test_do_eqstate_vs_oracle(method):
    c = started_case()
    c.pi["eqstate_method"] = method
    want = c.copy()
    oracle.bc_call(want, "do_eqstate")
    got = gpu_call(c, "do_eqstate")
    for k in ("rho", "buoy"):
        assert np.array_equal(got.f3[k], want.f3[k]), k


def test_gotm_parabolic_vs_oracle():
    c = started_case()
    c.pi["viscosity"] = 1
    c.pd.update(avmback=1e-5, avhback=3e-6)
    oracle.bc_call(c, "stresses_3d")  # taub of the current velocities
    want = c.copy()
    oracle.bc_call(want, "gotm_parabolic")
    got = gpu_call(c, "gotm")
    for k in ("num", "nuh", "tke", "eps"):
        assert np.array_equal(got.f3[k], want.f3[k]), k
    assert np.abs(want.f3["num"] - c.f3["num"]).max() > 1e-4  # the profile replaced the prescribed one


def radiation_inputs(c, seed=3):
    rng = np.random.default_rng(seed)
    g = c.grid
    wet = c.az >= 1
    c.pi["radiation"] = 1
    c.f2["swr"][...] = np.where(wet, rng.uniform(50.0, 350.0, g.shape2()), 0.0)
    c.f2["shf"][...] = np.where(wet, rng.uniform(-150.0, 100.0, g.shape2()), 0.0)
    c.f2["A"][...] = S.F32(0.58)
    c.f2["g1"][...] = S.F32(0.35)
    c.f2["g2"][...] = S.F32(23.0)
    return c


def test_sw_radiation_vs_oracle():
    c = radiation_inputs(started_case())
    want = c.copy()
    oracle.bc_call(want, "sw_radiation")
    got = gpu_call(c, "sw_radiation")
    assert field_err(got.f3["rad"], want.f3["rad"]) <= 1e-12
    assert float(np.abs(want.f3["rad"]).max()) > 50.0


@pytest.mark.parametrize("which", [2, 3], ids=["UNESCO80 + radiation", "Jackett06 + parabolic + reflection"])
def test_physics_options_vs_reference_fixture(which):
    """getm_time_loop with the options on, against the reference's own integrate_2d / integrate_3d
    executed on the same inputs (two macro steps): every field within 1e-12 of its scale."""
    import torch

    gold = dict(np.load(GOLD_PHYS[which]))
    c = load_case(gold)
    ctx, _ = make_ctx(c)
    st = BcDevice(c)
    ctx.time_loop(st, 1, 8)
    torch.cuda.synchronize()
    out = st.to_host(c.copy())
    bad = {}
    for k in gold_names(gold, "f2"):
        e = field_err(out.f2[k], gold["out_f2_" + k])
        if not e <= 1e-12:
            bad[k] = e
    for k in gold_names(gold, "f3"):
        e = field_err(out.f3[k], gold["out_f3_" + k])
        if not e <= 1e-12:
            bad[k] = e
    assert not bad, bad


@pytest.mark.parametrize("eos,visc,refl", [(3, 1, True), (2, 0, False)])
def test_physics_options_vs_oracle(eos, visc, refl):
    """The same options on a larger islands basin over 15 micro steps, FP64, against the oracle."""
    import torch

    c = radiation_inputs(S.baroclinic_case(nx=40, ny=28, kmax=10, recipe="islands", M=5, dt3=60.0, seed=11,
                                           land=0.3))
    c.pi.update(eqstate_method=eos, viscosity=visc)
    if refl:
        c.pd["swr_bot_refl_frac"] = 0.2
    if visc:
        c.pd.update(avmback=1e-5, avhback=2e-6)
    ref = c.copy()
    oracle.bc_steps(ref, 1, 15)
    ctx, _ = make_ctx(c)
    st = BcDevice(c)
    ctx.time_loop(st, 1, 15)
    torch.cuda.synchronize()
    out = st.to_host(c.copy())
    bad = {}
    for k in S.F2_NAMES:
        e = field_err(out.f2[k], ref.f2[k])
        if not e <= 1e-12:
            bad[k] = e
    for k in S.F3_NAMES:
        e = field_err(out.f3[k], ref.f3[k])
        if not e <= 1e-12:
            bad[k] = e
    assert not bad, bad


@pytest.mark.parametrize("eos,visc", [(3, 1), (2, 0)])
def test_physics_options_mixed_vs_fp64(eos, visc):
    """The mixed-precision step with the options on against the FP64 oracle after 10 macro steps
    (the bounds of the configured step)."""
    import torch

    c = radiation_inputs(S.baroclinic_case(nx=48, ny=40, kmax=10, recipe="islands", land=0.3, M=10, dt3=60.0,
                                           seed=6))
    c.pi.update(eqstate_method=eos, viscosity=visc)
    ref = c.copy()
    oracle.bc_steps(ref, 1, 100)
    c32 = c.copy(dtype3=np.float32)
    ctx, _ = make_ctx(c32)
    st = BcDevice(c32, dtype3=torch.float32)
    ctx.time_loop(st, 1, 100)
    torch.cuda.synchronize()
    out = st.to_host(c32.copy())
    errs = {k: field_err(out.f2[k], ref.f2[k]) for k in ("z", "U", "V")}
    errs.update({k: field_err(out.f3[k], ref.f3[k]) for k in ("uu", "vv", "T", "S", "num")})
    for k in ("T", "S"):
        assert errs[k] < 1e-5, errs
    for k in ("z", "U", "V", "uu", "vv", "num"):
        assert errs[k] < 1e-3, errs


def test_sealevel_nan_check_vs_reference():
    """getm_sealevel_nan_check against the reference's own classification of the same fields
    (tests/golden/reference_sealevel_nan.npz): count and last point."""
    from code_b200.getm import Context
    from code_b200.grid import Grid
    from helpers import dev

    g = dict(np.load(GOLD_NAN))
    nx, ny, kmax, dx, dy = g["meta"]
    ctx = Context(Grid(int(nx), int(ny), int(kmax), dx, dy))
    for q in range(3):
        n, last = ctx.sealevel_nan_check(dev(g[f"z{q}"]))
        assert n == int(g[f"count{q}"]), q
        if n:
            assert last == tuple(int(x) for x in g[f"last{q}"]), q


@pytest.mark.parametrize("chk", [1, -1, 3])
def test_time_loop_nan_sweep(chk):
    """sealevel_check in getm_time_loop: a NaN elevation is found by the sweep of a due micro step;
    sealevel_check > 0 makes the call return GETM_ERR_CHECK (the reference stops), < 0 only sets
    nan_warned; no finding without NaN."""
    import torch

    c = S.baroclinic_case(nx=24, ny=20, kmax=6, recipe="shelf", M=4, seed=5)
    c.pi["sealevel_check"] = chk
    ctx, _ = make_ctx(c)
    st = BcDevice(c)
    ctx.time_loop(st, 1, 8)  # clean: no finding
    assert st.ipar()["nan_warned"] == 0
    st.t["f2_z"][5, 7] = float("nan")
    raised = False
    try:
        ctx.time_loop(st, 9, 4)
    except GetmError as e:
        raised = True
        assert e.code == -4 and "NaN" in str(e)
    torch.cuda.synchronize()
    assert raised == (chk > 0)
    assert st.ipar()["nan_warned"] == 1


def _z_interpol_first_level_carries(c):
    """U columns whose first level (kmax-1) in ip_z_interpol.F90:83-125 finds no neighbour or own
    level to interpolate from (the search ends at level 1 or finds none) while below the surface
    test, so that it reads the buoyancy carried from the previous column in the loop order."""
    g = c.grid
    K = g.kmax

    def heights(Hb, h):
        z = np.empty_like(h)
        z[1] = -Hb + 0.5 * h[1]
        for k in range(2, K + 1):
            z[k] = z[k - 1] + 0.5 * (h[k - 1] + h[k])
        return z

    H = c.f2["H"]
    zz, zx = heights(H, c.f3["hn"]), heights(c.f2["HU"], c.f3["hun"])
    n = 0
    for j in range(2, 2 + g.ny):
        for i in range(2, 2 + g.nx):
            if c.au[j, i] < 1:
                continue
            x = zx[K - 1, j, i]
            kp = max([k for k in range(1, K + 1) if zz[k, j, i + 1] <= x], default=0)
            km = max([k for k in range(1, K + 1) if zz[k, j, i] <= x], default=0)
            n += (kp <= 1 or km <= 1) and x > max(-H[j, i + 1], -H[j, i])
    return n


def test_internal_pressure_z_interpol_carried_values():
    """ip_method 3 (Z_INTERPOL) on a steep islands bed (2-600 m, 5 levels): dozens of U columns
    start their downward loop without a level to interpolate from and read the buoyancies carried
    from the previous column of the reference's sequential loops (the device form finds them by a
    scan over the columns in loop order). FP64 bit for bit against the oracle, twice in a row on
    one context (the scan's scratch starts from the previous call's contents)."""
    import torch

    c = S.baroclinic_case(nx=40, ny=28, kmax=5, recipe="islands", M=5, dt3=60.0, seed=11, land=0.3, hmin=2.0,
                          hmax=600.0)
    c.pi["ip_method"] = 3
    assert _z_interpol_first_level_carries(c) >= 10
    want = c.copy()
    oracle.bc_call(want, "internal_pressure")
    ctx, _ = make_ctx(c)
    st = BcDevice(c, dtype3=torch.float64)
    for _ in range(2):
        ctx.internal_pressure(st)
        torch.cuda.synchronize()
        got = st.to_host(c.copy())
        for k in ("idpdx", "idpdy"):
            assert np.array_equal(got.f3[k], want.f3[k]), k


def test_internal_pressure_stelling_vankester_steep_bed():
    """ip_method 7 (STELLING_VANKESTER) on the steep islands bed (2-600 m, 5 levels): FP64 bit for
    bit against the oracle's sequential loops, twice in a row on one context."""
    import torch

    c = S.baroclinic_case(nx=40, ny=28, kmax=5, recipe="islands", M=5, dt3=60.0, seed=11, land=0.3, hmin=2.0,
                          hmax=600.0)
    c.pi["ip_method"] = 7
    want = c.copy()
    oracle.bc_call(want, "internal_pressure")
    ctx, _ = make_ctx(c)
    st = BcDevice(c, dtype3=torch.float64)
    for _ in range(2):
        ctx.internal_pressure(st)
        torch.cuda.synchronize()
        got = st.to_host(c.copy())
        for k in ("idpdx", "idpdy"):
            assert np.array_equal(got.f3[k], want.f3[k]), k
