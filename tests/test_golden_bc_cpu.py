"""The oracle's mode-split time loop against the reference's own integrate_2d / integrate_3d
(tests/golden/reference_mode_split.npz, made by tests/golden/make_golden_bc.py from the
reference's Fortran source): every 2D and 3D field of the state, bit for bit, after two macro
steps of four micro steps -- a closed basin, and (reference_mode_split_bdy.npz) a basin with open
boundaries of all four 2D types (update_2d_bdy, mirror_bdy_2d/3d)."""
import os

import numpy as np
import pytest

import oracle
from code_b200 import state as S
from code_b200.grid import Grid

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_mode_split.npz")
GOLD_BDY = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_mode_split_bdy.npz")


def load_case(gold, dtype3=np.float64):
    nx, ny, kmax, dx, dy = gold["meta"]
    c = S.BcCase(Grid(int(nx), int(ny), int(kmax), dx, dy), dtype3)
    for k in S.F2_NAMES:
        c.f2[k] = gold["in_f2_" + k].copy()
    for k in S.F3_NAMES:
        c.f3[k] = gold["in_f3_" + k].astype(dtype3)
    c.az, c.au, c.av, c.ax = (gold["in_" + k].copy() for k in ("az", "au", "av", "ax"))
    c.pd = dict(zip(S.PD_NAMES, (float(x) for x in gold["in_pd"])))
    c.pi = dict(zip(S.PI_NAMES, (int(x) for x in gold["in_pi"])))
    if "bdy_counts" in gold:
        sides, q = [], 0
        for n in gold["bdy_counts"]:
            sides.append([tuple(int(x) for x in row) for row in gold["bdy_seg"][q:q + int(n)]])
            q += int(n)
        b = S.OpenBoundaries(*sides, ramp=int(gold["bdy_ramp"]), amp=gold["bdy_amp"], phase=gold["bdy_phase"],
                             period=float(gold["bdy_period"]), data_v=gold["bdy_data_v"])
        c.bdy = b
    return c


@pytest.fixture(scope="module", params=["closed", "open boundaries"])
def gold(request):
    return dict(np.load(GOLD if request.param == "closed" else GOLD_BDY))


# fields the configuration never writes or reads (kept for the layout) are still compared
def test_time_loop_matches_reference(gold):
    c = load_case(gold)
    oracle.bc_steps(c, 1, 8)
    bad = []
    for k in S.F2_NAMES:
        if not np.array_equal(c.f2[k], gold["out_f2_" + k], equal_nan=True):
            bad.append((k, float(np.nanmax(np.abs(c.f2[k] - gold["out_f2_" + k])))))
    for k in S.F3_NAMES:
        if not np.array_equal(c.f3[k], gold["out_f3_" + k], equal_nan=True):
            bad.append((k, float(np.nanmax(np.abs(c.f3[k] - gold["out_f3_" + k])))))
    assert not bad, bad
