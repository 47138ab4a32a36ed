"""The oracle against the reference's own results (tests/golden/reference_hot_path.npz).

The fixtures hold outputs of the reference's Fortran routines executed from their source
(tests/golden/make_golden.py); every comparison here is exact (bit for bit)."""
import os

import numpy as np
import pytest

import oracle
from code_b200.cases import Case, derive_uvx
from code_b200.grid import Grid

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_hot_path.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def case_from(gold):
    nx, ny, kmax, dx, dy, dt = gold["case_meta"]
    g = Grid(int(nx), int(ny), int(kmax), dx, dy)
    c = Case(g, **{k[5:]: gold[k] for k in gold if k.startswith("case_") and k != "case_meta"})
    c.par["dt"] = float(dt)
    return c


def test_tridiagonal(gold):
    o = oracle.Oracle.__new__(oracle.Oracle)
    o.L = oracle.lib()
    for fi, lt in ((1, 9), (0, 9), (2, 5)):
        v = o.tridiagonal(9, fi, lt, *[gold[f"tri_in_{k}"].copy() for k in ("au", "bu", "cu", "du")])
        assert np.array_equal(v[fi:lt + 1], gold[f"tri_{fi}_{lt}"][fi:lt + 1])


def test_reconstruction(gold):
    c = case_from(gold)
    o = oracle.Oracle(c.grid)
    args = [gold[f"rec_in_{k}"] for k in ("cfl", "fuu", "fu", "fd")]
    for scheme in (1, 3, 4, 5, 6):
        assert np.array_equal(o.recon(scheme, *args), gold[f"rec_{scheme}"]), scheme


def test_masks(gold):
    c = case_from(gold)
    au, av, ax = derive_uvx(c["az"])
    assert np.array_equal(au, c["au"]) and np.array_equal(av, c["av"]) and np.array_equal(ax, c["ax"])
    o = oracle.Oracle(c.grid)
    mk = o.build_masks(*c.masks())
    for nm in ("updateH", "uflux", "vflux", "xflux", "uupdateU", "vupdateV"):
        assert np.array_equal(mk[nm], gold[f"mask_{nm}"]), nm


def test_do_advection_3d_all_configs(gold):
    c = case_from(gold)
    o = oracle.Oracle(c.grid)
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn")
    cfgs = gold["adv3d_configs"]
    assert len(cfgs) == 69
    for split, hs, vs, tag, AH in cfgs:
        split, hs, vs, tag = int(split), int(hs), int(vs), int(tag)
        f = c["f"].copy()
        h = np.zeros_like(f)
        a = np.zeros_like(f)
        o.do_advection_3d(c.masks(), c.par["dt"], f, *[c[n] for n in names], split, hs, vs, AH, tag, h, a, 1)
        key = f"adv3d_{split}_{hs}_{vs}_{tag}"
        assert np.array_equal(f, gold[key + "_f"]), key
        assert np.array_equal(h, gold[key + "_h"]), key
        assert np.array_equal(a, gold[key + "_a"]), key


def test_vertical_iterations(gold):
    c = case_from(gold)
    c["ww"] = gold["case_ww6"]
    o = oracle.Oracle(c.grid)
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn")
    for iters in (2, 4):
        f = c["f"].copy()
        h = np.zeros_like(f)
        a = np.zeros_like(f)
        warn = o.do_advection_3d(c.masks(), c.par["dt"], f, *[c[n] for n in names], 2, 6, 6, 0.0, 10, h, a, iters)
        assert np.array_equal(f, gold[f"adv3d_iter{iters}_f"])
        assert np.array_equal(h, gold[f"adv3d_iter{iters}_h"])
        assert np.array_equal(a, gold[f"adv3d_iter{iters}_a"])
        assert warn == int(gold[f"adv3d_iter{iters}_warn"][0])


@pytest.mark.parametrize("cn_name,cn", [("09", float(np.float32(0.9))), ("10", 1.0)])
def test_do_salinity(gold, cn_name, cn):
    """Three steps of the reference's do_salinity (advection P2_PDM HALFSPLIT + implicit diffusion
    with avmols = 1.1e-9 as a single-precision literal)."""
    c = case_from(gold)
    o = oracle.Oracle(c.grid)
    f = c["f"].copy()
    names = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn", "nuh")
    o.tracer_steps(c.masks(), 3, c.par["dt"], f, *[c[n] for n in names], 2, 6, 6, 0.0, cn,
                   float(np.float32(1.1e-9)))
    assert np.array_equal(f, gold[f"salt_{cn_name}"])
