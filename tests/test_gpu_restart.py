"""Hotstart through the C ABI: getm_restart_read (the restart file's fields into the device state,
then the reference's postinit_2d / postinit_3d re-initialisation) against the reference's own
routines executed on the same inputs (tests/golden/reference_hotstart.npz), FP64 bit for bit; and
getm_restart_write, whose output is the restart fields' interiors (the file's extent), FP64 and
FP32 (widened) states."""
import numpy as np
import pytest

from code_b200 import state as S
from code_b200.getm import BcDevice, restart_fields
from helpers import make_ctx
from test_golden_bc_cpu import GOLD_HOT, gold_names, hotstart_case

pytestmark = pytest.mark.gpu


def test_restart_read_matches_reference():
    import torch

    g = dict(np.load(GOLD_HOT))
    c, files = hotstart_case(g)
    ctx, _ = make_ctx(c)
    st = BcDevice(c)
    ctx.restart_read(st, 4, files)
    torch.cuda.synchronize()
    out = st.to_host(c.copy())
    for k in gold_names(g, "f2"):
        assert np.array_equal(out.f2[k], g["out_f2_" + k], equal_nan=True), k
    for k in gold_names(g, "f3"):
        assert np.array_equal(out.f3[k], g["out_f3_" + k], equal_nan=True), k


@pytest.mark.parametrize("dtype3", [np.float64, np.float32], ids=["fp64", "fp32"])
def test_restart_write_is_the_interior(dtype3):
    import torch

    c = S.baroclinic_case(nx=21, ny=17, kmax=6, recipe="islands", land=0.3, M=4, seed=3).copy(dtype3=dtype3)
    ctx, _ = make_ctx(c)
    st = BcDevice(c, dtype3=torch.float64 if dtype3 == np.float64 else torch.float32)
    ctx.time_loop(st, 1, 8)
    got = ctx.restart_write(st, 4)
    host = st.to_host(c.copy())
    i2, i3 = restart_fields(4)
    assert [S.F2_NAMES[q] for q in i2] == ["z", "zo", "U", "SlUx", "Slru", "V", "SlVx", "Slrv", "ssen", "ssun",
                                            "ssvn", "sseo", "ssuo", "ssvo", "Uinto", "Vinto"]
    assert [S.F3_NAMES[q] for q in i3] == ["uu", "vv", "ww", "uuEx", "vvEx", "tke", "eps", "num", "nuh", "hn", "T",
                                            "S"]
    for k, v in got.items():
        want = host.f2[k][2:-2, 2:-2] if k in host.f2 and v.ndim == 2 else host.f3[k][:, 2:-2, 2:-2]
        assert v.dtype == np.float64
        assert np.array_equal(v, np.asarray(want, np.float64)), k
    # read back into the same state: the water values come back unchanged, and postinit marks the
    # land (T = S = -9999, z = zo = -9999)
    ctx.restart_read(st, 4, got)
    again = ctx.restart_write(st, 4)
    wet = c.az[2:-2, 2:-2] >= 1
    for k in ("uu", "vv", "Uinto", "Vinto", "U", "V", "num"):
        assert np.array_equal(again[k][..., wet], got[k][..., wet]), k
    for k in ("T", "S"):
        assert np.array_equal(again[k][:, wet], got[k][:, wet]), k
        assert np.all(again[k][:, ~wet] == -9999.0), k
    assert np.all(again["z"][~wet] == -9999.0)
