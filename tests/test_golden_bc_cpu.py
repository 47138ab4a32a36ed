"""The oracle's mode-split time loop against the reference's own integrate_2d / integrate_3d
(tests/golden/reference_mode_split.npz, made by tests/golden/make_golden_bc.py from the
reference's Fortran source): every 2D and 3D field of the state, bit for bit, after two macro
steps of four micro steps -- a closed basin, (reference_mode_split_bdy.npz) a basin with open
boundaries of all four 2D types (update_2d_bdy, mirror_bdy_2d/3d), and
(reference_mode_split_ip{2,...,7}.npz) islands basins with the linear Blumberg-Mellor, z-interpolation, Stelling-van Kester, Song-Wright,
Chu-Fan and Shchepetkin-McWilliams internal pressure."""
import os

import numpy as np
import pytest

import oracle
from code_b200 import state as S
from code_b200.grid import Grid

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_mode_split.npz")
GOLD_BDY = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_mode_split_bdy.npz")
GOLD_IP = {m: os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"reference_mode_split_ip{m}.npz")
           for m in (2, 3, 4, 5, 6, 7)}
GOLD_IP2 = GOLD_IP[2]
GOLD_PHYS = {m: os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"reference_mode_split_phys{m}.npz")
             for m in (2, 3)}


def load_case(gold, dtype3=np.float64):
    nx, ny, kmax, dx, dy = gold["meta"]
    c = S.BcCase(Grid(int(nx), int(ny), int(kmax), dx, dy), dtype3)
    # fields and parameters added to the state after a fixture was written keep the case's zeros /
    # the reference's defaults (the options they belong to are off in such a fixture)
    for k in S.F2_NAMES:
        if "in_f2_" + k in gold:
            c.f2[k] = gold["in_f2_" + k].copy()
    for k in S.F3_NAMES:
        if "in_f3_" + k in gold:
            c.f3[k] = gold["in_f3_" + k].astype(dtype3)
    c.az, c.au, c.av, c.ax = (gold["in_" + k].copy() for k in ("az", "au", "av", "ax"))
    names_pd = [str(x) for x in gold["names_pd"]] if "names_pd" in gold else S.PD_NAMES
    names_pi = [str(x) for x in gold["names_pi"]] if "names_pi" in gold else S.PI_NAMES
    c.pd = dict(S.PARAM_DEFAULTS_PD)
    c.pd.update(zip(names_pd, (float(x) for x in gold["in_pd"])))
    c.pi = dict(S.PARAM_DEFAULTS_PI)
    c.pi.update(zip(names_pi, (int(x) for x in gold["in_pi"])))
    if "bdy_counts" in gold:
        sides, q = [], 0
        for n in gold["bdy_counts"]:
            sides.append([tuple(int(x) for x in row) for row in gold["bdy_seg"][q:q + int(n)]])
            q += int(n)
        b = S.OpenBoundaries(*sides, ramp=int(gold["bdy_ramp"]), amp=gold["bdy_amp"], phase=gold["bdy_phase"],
                             period=float(gold["bdy_period"]), data_v=gold["bdy_data_v"])
        c.bdy = b
    return c


def gold_names(gold, kind):
    """The fields of the state table that a fixture holds outputs of (fixtures written before a
    field was added to the table do not have it)."""
    names = S.F2_NAMES if kind == "f2" else S.F3_NAMES
    return [k for k in names if f"out_{kind}_{k}" in gold]


GOLDS = {"closed": GOLD, "open boundaries": GOLD_BDY, **{f"ip_method {m}": GOLD_IP[m] for m in (2, 3, 4, 5, 6, 7)},
         "radiation, UNESCO80": GOLD_PHYS[2], "radiation + bottom reflection, Jackett 2006, parabolic viscosity":
         GOLD_PHYS[3]}


@pytest.fixture(scope="module", params=list(GOLDS))
def gold(request):
    return dict(np.load(GOLDS[request.param]))


# fields the configuration never writes or reads (kept for the layout) are still compared
def test_time_loop_matches_reference(gold):
    c = load_case(gold)
    oracle.bc_steps(c, 1, 8)
    bad = []
    for k in gold_names(gold, "f2"):
        if not np.array_equal(c.f2[k], gold["out_f2_" + k], equal_nan=True):
            bad.append((k, float(np.nanmax(np.abs(c.f2[k] - gold["out_f2_" + k])))))
    for k in gold_names(gold, "f3"):
        if not np.array_equal(c.f3[k], gold["out_f3_" + k], equal_nan=True):
            bad.append((k, float(np.nanmax(np.abs(c.f3[k] - gold["out_f3_" + k])))))
    assert not bad, bad


@pytest.mark.parametrize("method", [2, 3, 4, 5, 6, 7])
def test_ip_method_fixture_differs_from_method_1(method):
    """Each internal-pressure fixture pins a method of its own: the oracle with Blumberg-Mellor (1)
    on the same inputs gives other internal pressure gradients."""
    gold = dict(np.load(GOLD_IP[method]))
    c = load_case(gold)
    assert c.pi["ip_method"] == method
    c.pi["ip_method"] = 1
    oracle.bc_steps(c, 1, 8)
    assert not np.array_equal(c.f3["idpdx"], gold["out_f3_idpdx"])
    assert not np.array_equal(c.f3["idpdy"], gold["out_f3_idpdy"])


GOLD_NAN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_sealevel_nan.npz")


def test_sealevel_nan_check_matches_reference():
    """sealevel_nan_check (sealevel.F90:172-314) in the oracle against the reference's own per-point
    classification (tests/golden/reference_sealevel_nan.npz): the number of interior elevations not
    below HUGE (NaN, +Inf, HUGE; not -Inf, subnormals or halo points) and the last of them in loop
    order."""
    g = dict(np.load(GOLD_NAN))
    nx, ny, kmax, dx, dy = g["meta"]
    grid = Grid(int(nx), int(ny), int(kmax), dx, dy)
    for q in range(3):
        n, last = oracle.sealevel_nan_check(grid, g[f"z{q}"])
        assert n == int(g[f"count{q}"]), q
        if n:
            assert last == tuple(int(x) for x in g[f"last{q}"]), q


def test_sealevel_check_stops_like_reference():
    """sealevel_check > 0 turns a NaN finding into an error, < 0 into a warning that also ends the
    checks (have_warned), as the reference's sealevel does on the same fields."""
    g = dict(np.load(GOLD_NAN))
    nx, ny, kmax, dx, dy = g["meta"]
    for q in range(3):
        for col, chk in ((0, 1), (1, -1)):
            c = S.baroclinic_case(nx=int(nx), ny=int(ny), kmax=int(kmax), recipe="islands", land=0.3, M=4, dt3=60.0,
                                  seed=5)
            c.f2["z"][...] = g[f"z{q}"]
            c.pd["dtm"] = 0.0
            c.pi["sealevel_check"] = chk
            stops = bool(g[f"stops{q}"][col])
            try:
                oracle.bc_call(c, "integrate_2d", 1)
                stopped = False
            except ValueError:
                stopped = True
            assert stopped == stops, (q, chk)
            assert c.pi["nan_warned"] == (1 if int(g[f"count{q}"]) > 0 else 0), (q, chk)


def test_native_oracle_build_is_bit_exact():
    """The -march=native build of the oracle (the one the benchmark times on the host cores) gives
    the reference's bits on every mode-split fixture, like the portable build (no contraction, no
    reassociation in either). Run in a child process, which selects that build."""
    import subprocess
    import sys

    code = (
        "import sys, numpy as np\n"
        "sys.path[:0] = ['.', 'tests']\n"
        "import oracle\n"
        "assert oracle.use_native_build()\n"
        "from test_golden_bc_cpu import GOLDS, gold_names, load_case\n"
        "for name, path in GOLDS.items():\n"
        "    g = dict(np.load(path)); c = load_case(g); oracle.bc_steps(c, 1, 8)\n"
        "    for k in gold_names(g, 'f2'): assert np.array_equal(c.f2[k], g['out_f2_' + k], equal_nan=True), (name, k)\n"
        "    for k in gold_names(g, 'f3'): assert np.array_equal(c.f3[k], g['out_f3_' + k], equal_nan=True), (name, k)\n"
        "print('ok')\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]


GOLD_HOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_hotstart.npz")


def hotstart_case(gold):
    """The fixture's state before the restart file is read, and the file's interiors {name: array}."""
    c = load_case(gold)
    files = {k[8:]: gold[k] for k in gold if k.startswith("file_f2_")}
    files.update({k[8:]: gold[k] for k in gold if k.startswith("file_f3_")})
    return c, files


def test_hotstart_postinit_matches_reference():
    """The oracle's hotstart re-initialisation (postinit_2d / postinit_3d with hotstart = .true.)
    after the restart file's interiors are read, against the reference's own routines on the same
    inputs (tests/golden/reference_hotstart.npz): every field bit for bit."""
    g = dict(np.load(GOLD_HOT))
    c, files = hotstart_case(g)
    for k, v in files.items():
        (c.f2 if k in c.f2 and v.ndim == 2 else c.f3)[k][..., 2:-2, 2:-2] = v
    oracle.bc_call(c, "hotstart_postinit", 4)
    for k in gold_names(g, "f2"):
        assert np.array_equal(c.f2[k], g["out_f2_" + k], equal_nan=True), k
    for k in gold_names(g, "f3"):
        assert np.array_equal(c.f3[k], g["out_f3_" + k], equal_nan=True), k
