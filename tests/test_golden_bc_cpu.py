"""The oracle's mode-split time loop against the reference's own integrate_2d / integrate_3d
(tests/golden/reference_mode_split.npz, made by tests/golden/make_golden_bc.py from the
reference's Fortran source): every 2D and 3D field of the state, bit for bit, after two macro
steps of four micro steps -- a closed basin, (reference_mode_split_bdy.npz) a basin with open
boundaries of all four 2D types (update_2d_bdy, mirror_bdy_2d/3d), and
(reference_mode_split_ip{2,4,5,6}.npz) islands basins with the linear Blumberg-Mellor, Song-Wright,
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
           for m in (2, 4, 5, 6)}
GOLD_IP2 = GOLD_IP[2]


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
    c.pi.setdefault("ip_method", 1)  # fixtures written before the parameter existed
    if "bdy_counts" in gold:
        sides, q = [], 0
        for n in gold["bdy_counts"]:
            sides.append([tuple(int(x) for x in row) for row in gold["bdy_seg"][q:q + int(n)]])
            q += int(n)
        b = S.OpenBoundaries(*sides, ramp=int(gold["bdy_ramp"]), amp=gold["bdy_amp"], phase=gold["bdy_phase"],
                             period=float(gold["bdy_period"]), data_v=gold["bdy_data_v"])
        c.bdy = b
    return c


GOLDS = {"closed": GOLD, "open boundaries": GOLD_BDY, **{f"ip_method {m}": GOLD_IP[m] for m in (2, 4, 5, 6)}}


@pytest.fixture(scope="module", params=list(GOLDS))
def gold(request):
    return dict(np.load(GOLDS[request.param]))


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


@pytest.mark.parametrize("method", [2, 4, 5, 6])
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
