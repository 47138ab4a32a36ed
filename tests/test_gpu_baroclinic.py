"""The CUDA mode-split step (getm_time_loop / getm_integrate_2d / getm_integrate_3d) against the
reference's own integrate_2d / integrate_3d (golden fixture) and against the oracle.

Tolerance (FP64): every field within 1e-12 of the reference, relative to the field's largest
magnitude. All arithmetic is evaluated in the reference's order without contraction; the one
source of difference is the natural logarithm of the log-law drag (bottom_friction.F90,
bottom_friction_3d.F90, slow_bottom_friction.F90), where the device's log and the host's libm
may differ in the last bit.
"""
import numpy as np
import pytest

import oracle
from code_b200 import state as S
from code_b200.getm import BcDevice
from helpers import make_ctx
from test_golden_bc_cpu import GOLD, GOLD_BDY, GOLD_IP, gold_names, load_case

pytestmark = pytest.mark.gpu


def field_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.nanmax(np.abs(b))), 1e-300)
    return float(np.nanmax(np.abs(a - b))) / scale


def compare(case_gpu, ref_f2, ref_f3, tol):
    worst = {}
    for k in ref_f2:
        worst[k] = field_err(case_gpu.f2[k], ref_f2[k])
    for k in ref_f3:
        worst[k] = field_err(case_gpu.f3[k], ref_f3[k])
    bad = {k: v for k, v in worst.items() if not v <= tol}
    return bad, worst


def run_gpu(c, n0, count, dtype3=None):
    import torch

    ctx, _ = make_ctx(c)
    if c.bdy is not None:
        ctx.set_open_boundaries(c.bdy)
    st = BcDevice(c, dtype3=dtype3)
    ctx.time_loop(st, n0, count)
    torch.cuda.synchronize()
    out = c.copy()
    st.to_host(out)
    return out, ctx


@pytest.mark.parametrize("path", [GOLD, GOLD_BDY] + [GOLD_IP[m] for m in (2, 3, 4, 5, 6, 7)],
                         ids=["closed", "open boundaries"] + [f"ip_method {m}" for m in (2, 3, 4, 5, 6, 7)])
def test_time_loop_vs_reference_fixture(path):
    gold = dict(np.load(path))
    c = load_case(gold)
    out, _ = run_gpu(c, 1, 8)
    bad, worst = compare(out, {k: gold["out_f2_" + k] for k in gold_names(gold, "f2")},
                         {k: gold["out_f3_" + k] for k in gold_names(gold, "f3")}, 1e-12)
    assert not bad, bad


@pytest.mark.parametrize("recipe,nx,ny,kmax", [("shelf", 40, 28, 10), ("islands", 48, 40, 8), ("flat", 33, 21, 6)])
def test_time_loop_vs_oracle(recipe, nx, ny, kmax):
    c = S.baroclinic_case(nx=nx, ny=ny, kmax=kmax, recipe=recipe, M=5, dt3=60.0, seed=11, land=0.3)
    ref = c.copy()
    oracle.bc_steps(ref, 1, 15)
    out, ctx = run_gpu(c, 1, 15)
    assert out.pi["ufirst2d"] == ref.pi["ufirst2d"] and out.pi["ufirst3d"] == ref.pi["ufirst3d"]
    bad, worst = compare(out, ref.f2, ref.f3, 1e-12)
    assert not bad, bad
    assert ctx.take_warnings() == 0


def test_barotropic_runtype_vs_oracle():
    """runtype 1 (barotropic only): the time loop runs no macro step (do_3d, integration.F90:106),
    the bottom friction renews the roughness zub/zvb every MM micro steps and Uint/Vint are not
    accumulated; FP64 against the oracle, and the 3D fields left as they were."""
    c = S.baroclinic_case(nx=48, ny=40, kmax=8, recipe="islands", M=5, dt3=60.0, seed=11, land=0.3)
    c.pi["runtype"] = 1
    ref = c.copy()
    oracle.bc_steps(ref, 1, 17)
    out, ctx = run_gpu(c, 1, 17)
    bad, worst = compare(out, ref.f2, ref.f3, 1e-12)
    assert not bad, bad
    for k in S.F3_NAMES:
        assert np.array_equal(out.f3[k], c.f3[k], equal_nan=True), k
    assert not np.array_equal(out.f2["zub"], c.f2["zub"])  # renewed
    assert ctx.take_warnings() == 0


@pytest.mark.parametrize("runtype", [1, 4])
def test_mixed_roughness_working_copies(runtype):
    """The mixed micro steps keep the bottom roughness as FP32 working copies: with runtype 1 the
    FP32 bottom friction renews it and the new values come back to the state (the fused and the
    separate launches give the same bits; within 1e-4 of the FP64 run, whose velocities the mixed
    ones follow to about that); with runtype 4 it is only read, and the state's FP64 roughness
    stays bit for bit what it was."""
    import torch

    from code_b200 import getm as G

    c = S.baroclinic_case(nx=77, ny=53, kmax=8, recipe="islands", land=0.3, M=5, dt3=60.0, seed=4)
    c.pi["runtype"] = runtype
    ref = c.copy()
    oracle.bc_steps(ref, 1, 23)
    c32 = c.copy(dtype3=np.float32)
    out = {}
    prev = G.set_fused_micro_step(True)
    try:
        for on in (True, False):
            G.set_fused_micro_step(on)
            out[on], _ = run_gpu(c32, 1, 23, dtype3=torch.float32)
    finally:
        G.set_fused_micro_step(prev)
    for k in S.F2_NAMES:
        assert np.array_equal(out[True].f2[k], out[False].f2[k], equal_nan=True), k
    for k in ("zub", "zvb"):
        if runtype == 1:
            assert field_err(out[True].f2[k], ref.f2[k]) <= 1e-4, k
            assert not np.array_equal(out[True].f2[k], c.f2[k]), k
        else:
            assert np.array_equal(out[True].f2[k], c.f2[k]), k


def tidal_shelf(nx=40, ny=28, kmax=10, M=5, period=900.0, seed=11):
    """The shelf configuration with its western side open and clamped to a tide (1 m amplitude;
    the period is shortened from M2 so that the test sees a full cycle), ramped over 40 micro
    steps."""
    g = S.Grid(nx, ny, kmax, 1000.0, 1000.0)
    b = S.OpenBoundaries(west=[(g.imin, g.jmin, g.jmax, S.CLAMPED)], ramp=40, amp=1.0, period=period)
    return S.baroclinic_case(nx=nx, ny=ny, kmax=kmax, recipe="shelf", M=M, dt3=60.0, seed=seed, bdy=b)


def test_open_boundary_tide_vs_oracle():
    c = tidal_shelf()
    ref = c.copy()
    oracle.bc_steps(ref, 1, 30)
    out, ctx = run_gpu(c, 1, 30)
    bad, worst = compare(out, ref.f2, ref.f3, 1e-12)
    assert not bad, bad
    # the boundary moved the sea surface
    assert np.abs(out.f2["z"][:, 2]).max() > 0.1


def test_open_boundary_data_from_host():
    """getm_set_bdy_data (fixed data, all four types) equals the oracle run with the same data."""
    g = S.Grid(30, 24, 6, 1000.0, 1000.0)
    b = S.OpenBoundaries(west=[(g.imin, g.jmin + 2, g.jmax - 2, S.CLAMPED)],
                         north=[(g.jmax, g.imin + 3, g.imax - 3, S.ZERO_GRADIENT)],
                         east=[(g.imax, g.jmin + 2, g.jmax - 2, S.SOMMERFELD)],
                         south=[(g.jmin, g.imin + 3, g.imax - 3, S.FLATHER_ELEV)], ramp=8)
    n = b.npoints()
    b.data = np.linspace(-0.2, 0.3, n)
    b.data_v = np.full(n, 0.01)
    c = S.baroclinic_case(nx=30, ny=24, kmax=6, recipe="shelf", M=4, seed=2, bdy=b)
    ref = c.copy()
    oracle.bc_steps(ref, 1, 12)
    out, _ = run_gpu(c, 1, 12)
    bad, worst = compare(out, ref.f2, ref.f3, 1e-12)
    assert not bad, bad


def test_integrate_entry_points_match_time_loop():
    """getm_integrate_2d + getm_integrate_3d called one by one equal getm_time_loop."""
    import torch

    c = S.baroclinic_case(nx=24, ny=20, kmax=6, recipe="shelf", M=3, seed=5)
    a, _ = run_gpu(c, 1, 6)
    ctx, _ = make_ctx(c)
    st = BcDevice(c)
    for n in range(1, 7):
        ctx.integrate_2d(st, n)
        if n % 3 == 0:
            ctx.integrate_3d(st, n)
    torch.cuda.synchronize()
    b = st.to_host(c.copy())
    for k in S.F2_NAMES:
        assert np.array_equal(a.f2[k], b.f2[k], equal_nan=True), k
    for k in S.F3_NAMES:
        assert np.array_equal(a.f3[k], b.f3[k], equal_nan=True), k


def test_mixed_precision_error_vs_fp64():
    """The mixed variant (3D fields FP32; 2D, Uint/Vint and vertical sums FP64) against the FP64
    oracle after 10 macro steps of the tidally forced shelf: per-field error relative to the
    field's scale (stated bounds)."""
    import torch

    c = tidal_shelf(nx=48, ny=40, kmax=10, M=10, period=3000.0, seed=3)
    ref = c.copy()
    oracle.bc_steps(ref, 1, 100)
    out, _ = run_gpu(c.copy(dtype3=np.float32), 1, 100, dtype3=torch.float32)
    errs = {k: field_err(out.f2[k], ref.f2[k]) for k in ("z", "U", "V")}
    errs.update({k: field_err(out.f3[k], ref.f3[k]) for k in ("uu", "vv", "T", "S")})
    for k in ("T", "S"):
        assert errs[k] < 1e-5, errs
    for k in ("z", "U", "V", "uu", "vv"):
        assert errs[k] < 1e-3, errs


def test_mixed_closed_basin_error_vs_fp64():
    """The mixed variant on a closed basin -- its micro steps run on the FP32 working copies of the
    barotropic fields (elevation and Uint/Vint FP64) -- against the FP64 oracle after 10 macro
    steps: per-field error relative to the field's scale (stated bounds)."""
    import torch

    c = S.baroclinic_case(nx=48, ny=40, kmax=10, recipe="islands", land=0.3, M=10, dt3=60.0, seed=6)
    ref = c.copy()
    oracle.bc_steps(ref, 1, 100)
    out, _ = run_gpu(c.copy(dtype3=np.float32), 1, 100, dtype3=torch.float32)
    errs = {k: field_err(out.f2[k], ref.f2[k]) for k in ("z", "U", "V")}
    errs.update({k: field_err(out.f3[k], ref.f3[k]) for k in ("uu", "vv", "T", "S")})
    for k in ("T", "S"):
        assert errs[k] < 1e-5, errs
    for k in ("z", "U", "V", "uu", "vv"):
        assert errs[k] < 1e-3, errs


def test_mixed_time_loop_split_calls_match():
    """The FP32 working copies are written back at the end of each getm_time_loop call and refilled
    at the start of the next: four calls of 10 micro steps equal one call of 40, bit for bit."""
    import torch

    c = S.baroclinic_case(nx=40, ny=36, kmax=8, recipe="islands", land=0.3, M=5, dt3=60.0, seed=2)
    c = c.copy(dtype3=np.float32)
    a, _ = run_gpu(c, 1, 40, dtype3=torch.float32)
    ctx, _ = make_ctx(c)
    st = BcDevice(c, dtype3=torch.float32)
    for n0 in (1, 11, 21, 31):
        ctx.time_loop(st, n0, 10)
    torch.cuda.synchronize()
    b = st.to_host(c.copy())
    for k in S.F2_NAMES:
        assert np.array_equal(a.f2[k], b.f2[k], equal_nan=True), k
    for k in S.F3_NAMES:
        assert np.array_equal(a.f3[k], b.f3[k], equal_nan=True), k


def rms_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.nanmax(np.abs(b))), 1e-300)
    return float(np.sqrt(np.nanmean((a - b) ** 2))) / scale


def test_mixed_from_moving_state_vs_fp64():
    """The mixed variant started from moving water whose stored Coriolis terms are zero (the
    rotation recipe: U, V from a solid-body rotation, fU = fV = 0): the first velocity update of a
    call reads the stored term, as the reference's umomentum / vmomentum do, so the mixed run
    stays within FP32 rounding of the FP64 oracle (RMS over the field, relative to the field's
    scale; stated bounds) after 30 macro steps."""
    import torch

    c = S.baroclinic_case(nx=96, ny=96, kmax=12, recipe="rotation", dx=500.0, M=10, dt3=60.0, seed=3)
    assert np.abs(c.f2["U"]).max() > 1.0 and np.abs(c.f2["fU"]).max() == 0.0
    ref = c.copy()
    oracle.bc_steps(ref, 1, 300)
    out, _ = run_gpu(c.copy(dtype3=np.float32), 1, 300, dtype3=torch.float32)
    rms = {k: rms_err(out.f2[k], ref.f2[k]) for k in ("z", "U", "V")}
    rms.update({k: rms_err(out.f3[k], ref.f3[k]) for k in ("uu", "vv", "T")})
    big = {k: field_err(out.f2[k], ref.f2[k]) for k in ("z", "U", "V")}
    for k, v in rms.items():
        assert v < 1e-5, (rms, big)
    for k, v in big.items():
        assert v < 2e-4, (rms, big)


@pytest.mark.parametrize("recipe,nx,ny", [("islands", 77, 53), ("rotation", 64, 48)])
def test_mixed_kernel_forms_agree(recipe, nx, ny):
    """The mixed time loop with the vectorised kernels (the default: float4-lane sweeps, vectorised
    sigma heights, equation of state and momentum-advection inputs) and with the tile / scalar
    kernels (getm_set_vector_sweeps(0)) gives the same bits: both evaluate every cell's operations
    in the same order with the same rounding."""
    import torch

    from code_b200 import getm as G

    if recipe == "islands":
        c = S.baroclinic_case(nx=nx, ny=ny, kmax=8, recipe=recipe, land=0.3, M=5, dt3=60.0, seed=4)
    else:
        c = S.baroclinic_case(nx=nx, ny=ny, kmax=8, recipe=recipe, dx=500.0, M=5, dt3=60.0, seed=4)
    c = c.copy(dtype3=np.float32)
    out = {}
    prev = G.set_vector_sweeps(True)
    try:
        for on in (True, False):
            G.set_vector_sweeps(on)
            out[on], _ = run_gpu(c, 1, 20, dtype3=torch.float32)
    finally:
        G.set_vector_sweeps(prev)
    for k in S.F2_NAMES:
        assert np.array_equal(out[True].f2[k], out[False].f2[k], equal_nan=True), k
    for k in S.F3_NAMES:
        assert np.array_equal(out[True].f3[k], out[False].f3[k], equal_nan=True), k


@pytest.mark.parametrize("count", [20, 23])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_fused_micro_step_forms_agree(prec, count):
    """getm_time_loop with the fused micro-step launches (the default: sealevel + depth_update in
    one launch with the elevations alternating between z and zo; the mixed step's bottom friction
    inside its momentum-advection kernels) and with the separate launches
    (getm_set_fused_micro_step(0)) gives the same bits in every field, z and zo included -- after
    an even and an odd number of micro steps."""
    import torch

    from code_b200 import getm as G

    c = S.baroclinic_case(nx=77, ny=53, kmax=8, recipe="islands", land=0.3, M=5, dt3=60.0, seed=4)
    if prec == "mixed":
        c = c.copy(dtype3=np.float32)
    out = {}
    prev = G.set_fused_micro_step(True)
    try:
        for on in (True, False):
            G.set_fused_micro_step(on)
            out[on], _ = run_gpu(c, 1, count, dtype3=torch.float32 if prec == "mixed" else None)
    finally:
        G.set_fused_micro_step(prev)
    for k in S.F2_NAMES:
        assert np.array_equal(out[True].f2[k], out[False].f2[k], equal_nan=True), k
    for k in S.F3_NAMES:
        assert np.array_equal(out[True].f3[k], out[False].f3[k], equal_nan=True), k


@pytest.mark.parametrize("method", [2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("recipe", ["shelf", "islands"])
def test_ip_method_vs_oracle(recipe, method):
    """The other internal pressure methods -- linear Blumberg-Mellor (2), z-interpolation (3),
    Stelling-van Kester (7), Song-Wright (4), Chu-Fan
    (5), Shchepetkin-McWilliams (6) -- through getm_time_loop against the oracle, FP64, 1e-12 of
    each field's scale."""
    c = S.baroclinic_case(nx=40, ny=28, kmax=10, recipe=recipe, M=5, dt3=60.0, seed=11, land=0.3)
    c.pi["ip_method"] = method
    ref = c.copy()
    oracle.bc_steps(ref, 1, 15)
    out, ctx = run_gpu(c, 1, 15)
    bad, worst = compare(out, ref.f2, ref.f3, 1e-12)
    assert not bad, bad
    assert ctx.take_warnings() == 0


@pytest.mark.parametrize("method", [2, 3, 4, 5, 6, 7])
def test_ip_method_mixed_error_vs_fp64(method):
    """The mixed variant with internal pressure method 2, 4, 5 or 6 against the FP64 oracle after 10
    macro steps of the islands basin (the bounds of the Blumberg-Mellor case)."""
    import torch

    c = S.baroclinic_case(nx=48, ny=40, kmax=10, recipe="islands", land=0.3, M=10, dt3=60.0, seed=6)
    c.pi["ip_method"] = method
    ref = c.copy()
    oracle.bc_steps(ref, 1, 100)
    out, _ = run_gpu(c.copy(dtype3=np.float32), 1, 100, dtype3=torch.float32)
    errs = {k: field_err(out.f2[k], ref.f2[k]) for k in ("z", "U", "V")}
    errs.update({k: field_err(out.f3[k], ref.f3[k]) for k in ("uu", "vv", "T", "S")})
    for k in ("T", "S"):
        assert errs[k] < 1e-5, errs
    for k in ("z", "U", "V", "uu", "vv"):
        assert errs[k] < 1e-3, errs


@pytest.mark.parametrize("method,code", [(0, "GETM_ERR_ARG"), (8, "GETM_ERR_ARG")])
def test_ip_method_not_provided_is_refused(method, code):
    """Invalid ids are
    refused with an error code before any work (the reference stops on an invalid ip_method,
    internal_pressure.F90:166-167)."""
    from code_b200 import getm as G

    c = S.baroclinic_case(nx=16, ny=12, kmax=4, recipe="shelf", M=2, seed=1)
    c.pi["ip_method"] = method
    ctx, _ = make_ctx(c)
    st = BcDevice(c)
    with pytest.raises(G.GetmError) as e:
        ctx.time_loop(st, 1, 2)
    assert G.ERRORS[e.value.code] == code


def test_ip_method6_independent_of_scratch_history():
    """Shchepetkin-McWilliams internal pressure (method 6) reads the pressure-point heights of land
    columns next to water faces; those stay zero (as the reference's zz array does), whatever an
    earlier call left in the context's scratch. A mixed run on a context that first ran the FP64
    step (whose scratch arrays overlap the FP32 ones at other offsets) equals the same mixed run on
    a fresh context, bit for bit."""
    import torch

    c = S.baroclinic_case(nx=40, ny=28, kmax=10, recipe="islands", M=5, dt3=60.0, seed=11, land=0.3)
    c.pi["ip_method"] = 6
    c32 = c.copy(dtype3=np.float32)
    ctx, _ = make_ctx(c)
    st64 = BcDevice(c)
    ctx.time_loop(st64, 1, 10)
    st = BcDevice(c32, dtype3=torch.float32)
    ctx.time_loop(st, 1, 10)
    torch.cuda.synchronize()
    a = st.to_host(c32.copy())
    b, _ = run_gpu(c32, 1, 10, dtype3=torch.float32)
    for k in S.F3_NAMES:
        assert np.array_equal(a.f3[k], b.f3[k], equal_nan=True), k
    for k in S.F2_NAMES:
        assert np.array_equal(a.f2[k], b.f2[k], equal_nan=True), k


def _range_err(a, b, wet):
    m = np.broadcast_to(wet[None], b.shape).copy()
    m[0] = False
    a = np.asarray(a, np.float64)[m]
    b = np.asarray(b, np.float64)[m]
    return float(np.abs(a - b).max()) / float(b.max() - b.min())


def test_compensated_tracer_storage_keeps_small_increments():
    """The mixed step's temperature on 15 C plus a unit anomaly (the rotation recipe): with plain
    FP32 storage the increments below half an ulp of 15 C are lost at every sweep, and after 40
    macro steps the error against the FP64 oracle, relative to the field's range, is several times
    that of the compensated storage (T + Tlo), which stays below 1e-5 of the range."""
    import torch

    c = S.baroclinic_case(nx=96, ny=96, kmax=12, recipe="rotation", dx=500.0, M=10, dt3=60.0, seed=3, t_noise=1e-3)
    ref = c.copy()
    oracle.bc_steps(ref, 1, 400)
    wet = c.az == 1
    errs = {}
    for comp in (True, False):
        c32 = c.copy(dtype3=np.float32)
        ctx, _ = make_ctx(c32)
        st = BcDevice(c32, dtype3=torch.float32, compensated=comp)
        ctx.time_loop(st, 1, 400)
        torch.cuda.synchronize()
        out = st.to_host(c32.copy())
        errs[comp] = _range_err(out.f3["T"], ref.f3["T"], wet)
    assert errs[True] < 1e-5, errs
    assert errs[False] > 3 * errs[True], errs
