"""Parity of the CUDA advection / diffusion path with the oracle (FP64: bit-exact).

The FP64 kernels are built without FMA contraction and keep the reference's expression order,
so every cell must equal the oracle's value exactly (tolerance 0). FP32 results are compared
with the FP64 oracle within a stated relative tolerance.
"""
import numpy as np
import pytest

import oracle
from code_b200 import cases
from code_b200 import getm as G
from helpers import dev, host, make_ctx, max_abs, rel_err

pytestmark = pytest.mark.gpu

SCHEMES = [G.UPSTREAM, G.P2, G.SUPERBEE, G.MUSCL, G.P2_PDM]


# 37 x 29: rows of 41 cells (the tile sweeps); 44 x 30: rows of 48 cells, every row and level on a
# 16-byte boundary (the vectorised sweeps)
@pytest.fixture(scope="module", params=[(37, 29), (44, 30)], ids=["tile", "vec"])
def rc(request):
    nx, ny = request.param
    c = cases.random_case(nx=nx, ny=ny, kmax=9, seed=3)
    ctx, m = make_ctx(c)
    return c, ctx, m, oracle.Oracle(c.grid)


def _grid_masks(o, c, tag):
    mk = o.build_masks(*c.masks())
    if tag == G.U_TAG:
        return mk["uflux_U"], mk["xflux"], mk["uupdateU"], mk["uflux"], mk["uflux"]
    if tag == G.V_TAG:
        return mk["xflux"], mk["vflux_V"], mk["vflux"], mk["vupdateV"], mk["vflux"]
    return mk["uflux"], mk["vflux"], mk["updateH"], mk["updateH"], mk["updateH"]


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("dirn", ["u", "v"])
@pytest.mark.parametrize("aliased", [True, False])
def test_adv_split_h_bitexact(rc, scheme, dirn, aliased):
    c, ctx, m, o = rc
    g = c.grid
    k = 3
    f = c["f"][k].copy()
    fi = f.copy() if aliased else c["f"][k + 1].copy()
    Di = c["ho"][k].copy()
    adv = np.zeros_like(f)
    vel = c["uu" if dirn == "u" else "vv"][k].copy()
    hv = c["hun" if dirn == "u" else "hvn"][k].copy()
    uf, vf, uup, vup, _ = _grid_masks(o, c, G.H_TAG)
    mflux, mupd = (uf, uup) if dirn == "u" else (vf, vup)
    AH = 7.5 if scheme == G.MUSCL else 0.0
    # oracle
    of, ofi, oDi, oadv = f.copy(), fi.copy(), Di.copy(), adv.copy()
    if aliased:
        ofi = of
    fn = o.adv_split_u if dirn == "u" else o.adv_split_v
    fn(c.par["dt"], of, ofi, oDi, oadv, vel, hv, 0.5, scheme, AH, mflux, mupd)
    # gpu
    tf = dev(f)
    tfi = tf if aliased else dev(fi)
    tDi, tadv = dev(Di), dev(adv)
    gfn = ctx.adv_split_u if dirn == "u" else ctx.adv_split_v
    gfn(c.par["dt"], tf, tfi, tDi, tadv, dev(vel), dev(hv), 0.5, scheme, AH, dev(mflux), dev(mupd), nk=1)
    assert np.array_equal(host(tfi), ofi)
    assert np.array_equal(host(tDi), oDi)
    assert np.array_equal(host(tadv), oadv)


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("tag", [G.H_TAG, G.W_TAG])
def test_adv_split_w_bitexact(rc, scheme, tag):
    c, ctx, m, o = rc
    dt = c.par["dt"]
    f = c["f"].copy()
    hi = c["ho"].copy()
    adv = np.zeros_like(f)
    az = c["az"]
    of, ohi, oadv = f.copy(), hi.copy(), adv.copy()
    o.adv_split_w(dt, of, of, ohi, oadv, c["ww"], 1.0, scheme, tag, az, 1)
    tf, thi, tadv = dev(f), dev(hi), dev(adv)
    ctx.adv_split_w(dt, tf, tf, thi, tadv, dev(c["ww"]), 1.0, scheme, tag, m[0], 1)
    assert np.array_equal(host(tf), of)
    assert np.array_equal(host(thi), ohi)
    assert np.array_equal(host(tadv), oadv)


@pytest.mark.parametrize("scheme", [G.UPSTREAM, G.SUPERBEE, G.P2_PDM])
def test_adv_split_w_iterations(rc, scheme):
    """adv_ver_iterations > 1 with Courant numbers up to ~3 (adv_split_w.F90:211-246)."""
    c, ctx, m, o = rc
    dt = c.par["dt"]
    f = c["f"].copy()
    hi = c["ho"].copy()
    ww = c["ww"] * 6.0
    adv = np.zeros_like(f)
    of, ohi, oadv = f.copy(), hi.copy(), adv.copy()
    nwarn_o = o.adv_split_w(dt, of, of, ohi, oadv, ww, 1.0, scheme, G.H_TAG, c["az"], 2)
    tf, thi, tadv = dev(f), dev(hi), dev(adv)
    ctx.take_warnings()
    ctx.adv_split_w(dt, tf, tf, thi, tadv, dev(ww), 1.0, scheme, G.H_TAG, m[0], 2)
    assert ctx.take_warnings() == nwarn_o
    assert np.array_equal(host(tf), of)
    assert np.array_equal(host(thi), ohi)
    assert np.array_equal(host(tadv), oadv)


@pytest.mark.parametrize("split", [G.NOSPLIT, G.FULLSPLIT, G.HALFSPLIT, G.HVSPLIT])
@pytest.mark.parametrize("hs,vs", [(G.SUPERBEE, G.SUPERBEE), (G.P2_PDM, G.P2_PDM), (G.UPSTREAM, G.MUSCL),
                                   (G.P2, G.UPSTREAM), (G.MUSCL, G.NOADV), (G.NOADV, G.P2_PDM)])
@pytest.mark.parametrize("tag", [G.H_TAG, G.U_TAG, G.V_TAG])
def test_do_advection_3d_bitexact(rc, split, hs, vs, tag):
    c, ctx, m, o = rc
    if vs == G.NOADV and split == G.HVSPLIT:
        pytest.skip("reference stops: do_advection has no HVSPLIT")
    dt = c.par["dt"]
    AH = 3.0 if hs == G.MUSCL else 0.0
    args = [c[n] for n in ("uu", "vv", "ww", "hun", "hvn", "ho", "hn")]
    of = c["f"].copy()
    ohires = np.zeros_like(of)
    oadv = np.zeros_like(of)
    o.do_advection_3d(c.masks(), dt, of, *args, split, hs, vs, AH, tag, ohires, oadv, 1)
    tf = dev(c["f"])
    th, ta = dev(np.zeros_like(of)), dev(np.zeros_like(of))
    ctx.do_advection_3d(dt, tf, *[dev(a) for a in args], split, hs, vs, AH, tag, th, ta, 1)
    assert np.array_equal(host(tf), of)
    assert np.array_equal(host(th), ohires)
    assert np.array_equal(host(ta), oadv)


def test_do_advection_3d_invalid(rc):
    c, ctx, m, o = rc
    args = [dev(c[n]) for n in ("uu", "vv", "ww", "hun", "hvn", "ho", "hn")]
    tf = dev(c["f"])
    with pytest.raises(G.GetmError) as e:
        ctx.do_advection_3d(1.0, tf, *args, 7, G.SUPERBEE, G.SUPERBEE, 0.0, G.H_TAG)
    assert e.value.code == -1
    with pytest.raises(G.GetmError):
        ctx.do_advection_3d(1.0, tf, *args, G.HALFSPLIT, G.SUPERBEE, G.SUPERBEE, 0.0, 99)
    with pytest.raises(G.GetmError) as e:
        ctx.do_advection_3d(1.0, tf, *args, G.HALFSPLIT, G.FCT, G.SUPERBEE, 0.0, G.H_TAG)
    assert e.value.code == -3


@pytest.mark.parametrize("with_src", [False, True])
@pytest.mark.parametrize("cnpar", [0.9, 1.0, 0.5])
def test_tracer_vdiff_bitexact(rc, with_src, cnpar):
    c, ctx, m, o = rc
    dt = c.par["dt"]
    S = c["f"].copy()
    src = np.random.default_rng(9).normal(size=S.shape) * 1e-3 if with_src else None
    cn = float(np.float32(cnpar))  # the reference's default 0.9 is a single-precision literal
    o.tracer_vdiff(dt, cn, 1.1e-9, S, c["hn"], c["nuh"], c["az"], src)
    tS = dev(c["f"])
    ctx.tracer_vdiff(dt, cn, 1.1e-9, tS, dev(c["hn"]), dev(c["nuh"]), m[0], dev(src) if with_src else None)
    assert np.array_equal(host(tS), S)


@pytest.mark.parametrize("fi,lt", [(1, 9), (0, 9), (2, 5)])
def test_tridiagonal_columns_bitexact(rc, fi, lt):
    c, ctx, m, o = rc
    rng = np.random.default_rng(11)
    kmax, ncol = 9, 300
    au = rng.uniform(-1, 0, (kmax + 1, ncol))
    cu = rng.uniform(-1, 0, (kmax + 1, ncol))
    bu = 2.5 + rng.uniform(0, 1, (kmax + 1, ncol))
    du = rng.normal(size=(kmax + 1, ncol))
    want = np.zeros((kmax + 1, ncol))
    for col in range(ncol):
        v = o.tridiagonal(kmax, fi, lt, *(np.ascontiguousarray(a[:, col]) for a in (au, bu, cu, du)))
        want[fi:lt + 1, col] = v[fi:lt + 1]
    tv = dev(np.zeros((kmax + 1, ncol)))
    ctx.tridiagonal(kmax, fi, lt, dev(au), dev(bu), dev(cu), dev(du), tv)
    assert np.array_equal(host(tv), want)


def test_tracer_rotation_200_steps():
    """128x128x20 rotation case, 200 FP64 steps: cell-wise equal to the oracle (<= 1e-12 asked,
    0 obtained) and tracer content conserved to round-off."""
    c = cases.tracer_rotation()
    p = c.par
    o = oracle.Oracle(c.grid)
    ctx, m = make_ctx(c)
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    of = c["f"].copy()
    o.tracer_steps(c.masks(), 200, p["dt"], of, *[c[n] for n in names], p["split"], p["hscheme"], p["vscheme"],
                   p["AH"], p["cnpar"], p["avmol"])
    tf = dev(c["f"])
    dv = [dev(c[n]) for n in names]
    m0 = ctx.tracer_content(tf, dv[6], m[0])
    for _ in range(200):
        ctx.tracer_step(p["dt"], tf, *dv, p["split"], p["hscheme"], p["vscheme"], p["AH"], p["cnpar"], p["avmol"])
    out = host(tf)
    assert rel_err(out, of, floor=1e-300) <= 1e-12
    assert np.array_equal(out, of)
    m1 = ctx.tracer_content(tf, dv[6], m[0])
    assert abs(m1 - m0) / abs(m0) < 1e-13
    om = o.tracer_content(of, c["hn"], c["az"])
    assert abs(m1 - om) / abs(om) < 1e-15


def test_tracer_rotation_fp32_error():
    """FP32 tracer step against the FP64 oracle after 200 steps: max error relative to the
    field's amplitude (1) stays below 1e-5."""
    c = cases.tracer_rotation()
    p = c.par
    o = oracle.Oracle(c.grid)
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    of = c["f"].copy()
    o.tracer_steps(c.masks(), 200, p["dt"], of, *[c[n] for n in names], p["split"], p["hscheme"], p["vscheme"],
                   p["AH"], p["cnpar"], p["avmol"])
    ctx, m = make_ctx(c)
    tf = dev(c["f"].astype(np.float32))
    dv = [dev(c[n].astype(np.float32)) for n in names]
    for _ in range(200):
        ctx.tracer_step(float(p["dt"]), tf, *dv, p["split"], p["hscheme"], p["vscheme"], 0.0, 1.0, 0.0)
    err = max_abs(host(tf), of)
    assert err < 1e-5, err


def test_tracer_content_and_check(rc):
    c, ctx, m, o = rc
    tf, th = dev(c["f"]), dev(c["hn"])
    got = ctx.tracer_content(tf, th, m[0])
    want = o.tracer_content(c["f"], c["hn"], c["az"])
    assert abs(got - want) <= 1e-14 * abs(want) + 1e-12
    inner = c["f"][:, 2:-2, 2:-2]
    wet = (c["az"][2:-2, 2:-2] > 0)[None].repeat(inner.shape[0], 0)
    lo, hi = -1.0, 1.0
    want_n = int((((inner < lo) | (inner > hi)) & wet).sum())
    assert ctx.check_3d_fields(tf, m[0], lo, hi) == want_n


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("hs", [G.UPSTREAM, G.SUPERBEE, G.P2_PDM])
def test_vector_and_tile_sweeps_agree(dtype, hs):
    """The vectorised sweeps (FP32: u and v; FP64: v on two-cell lanes) and the tile sweeps give
    identical results (bit for bit), tracer step with record tape included."""
    import torch

    c = cases.random_case(nx=60, ny=45, kmax=7, seed=11)
    ctx, m = make_ctx(c)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    args = [dev(c[n]).to(tdt) for n in ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")]
    out = {}
    prev = G.set_vector_sweeps(True)
    try:
        for on in (True, False):
            G.set_vector_sweeps(on)
            f = dev(c["f"]).to(tdt)
            for _ in range(3):
                ctx.tracer_step(c.par["dt"], f, *args, G.HALFSPLIT, hs, hs, 0.0, 1.0, 0.0)
            ft = dev(c["f"]).to(tdt)
            tape = ctx.tape(tdt)
            tape[0].zero_()
            tape[1].zero_()
            ctx.tracer_step_record(c.par["dt"], ft, *args, G.HALFSPLIT, hs, hs, 0.0, 1.0, 0.0, tape)
            out[on] = (host(f), host(ft), host(tape[0]), host(tape[1]))
    finally:
        G.set_vector_sweeps(prev)
    for a, b in zip(out[True], out[False]):
        assert np.array_equal(a, b)
