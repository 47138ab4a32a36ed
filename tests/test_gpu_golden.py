"""The CUDA path against the reference's own results (tests/golden/reference_hot_path.npz),
bit for bit in FP64: every do_advection_3d configuration, the vertical sub-iterations and three
steps of do_salinity (advection + implicit vertical diffusion)."""
import numpy as np
import pytest

from code_b200 import getm as G
from helpers import dev, host, make_ctx
from test_golden_cpu import case_from, gold  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu

NAMES = ("uu", "vv", "ww", "hun", "hvn", "ho", "hn")


def test_do_advection_3d_all_configs(gold):  # noqa: F811
    c = case_from(gold)
    ctx, m = make_ctx(c)
    dv = [dev(c[n]) for n in NAMES]
    for split, hs, vs, tag, AH in gold["adv3d_configs"]:
        split, hs, vs, tag = int(split), int(hs), int(vs), int(tag)
        f = dev(c["f"])
        h = dev(np.zeros_like(c["f"]))
        a = dev(np.zeros_like(c["f"]))
        ctx.do_advection_3d(c.par["dt"], f, *dv, split, hs, vs, float(AH), tag, h, a, 1)
        key = f"adv3d_{split}_{hs}_{vs}_{tag}"
        assert np.array_equal(host(f), gold[key + "_f"]), key
        assert np.array_equal(host(h), gold[key + "_h"]), key
        assert np.array_equal(host(a), gold[key + "_a"]), key


def test_vertical_iterations(gold):  # noqa: F811
    c = case_from(gold)
    c["ww"] = gold["case_ww6"]
    ctx, m = make_ctx(c)
    dv = [dev(c[n]) for n in NAMES]
    for iters in (2, 4):
        f = dev(c["f"])
        h = dev(np.zeros_like(c["f"]))
        a = dev(np.zeros_like(c["f"]))
        ctx.take_warnings()
        ctx.do_advection_3d(c.par["dt"], f, *dv, G.HALFSPLIT, G.P2_PDM, G.P2_PDM, 0.0, G.H_TAG, h, a, iters)
        assert np.array_equal(host(f), gold[f"adv3d_iter{iters}_f"])
        assert np.array_equal(host(h), gold[f"adv3d_iter{iters}_h"])
        assert np.array_equal(host(a), gold[f"adv3d_iter{iters}_a"])
        assert ctx.take_warnings() == int(gold[f"adv3d_iter{iters}_warn"][0])


@pytest.mark.parametrize("cn_name,cn", [("09", float(np.float32(0.9))), ("10", 1.0)])
def test_do_salinity(gold, cn_name, cn):  # noqa: F811
    c = case_from(gold)
    ctx, m = make_ctx(c)
    f = dev(c["f"])
    dv = [dev(c[n]) for n in NAMES + ("nuh",)]
    for _ in range(3):
        ctx.tracer_step(c.par["dt"], f, *dv, G.HALFSPLIT, G.P2_PDM, G.P2_PDM, 0.0, cn, float(np.float32(1.1e-9)))
    assert np.array_equal(host(f), gold[f"salt_{cn_name}"])
