"""getm_tracer_vdiff_noalloc: the context-free vertical-diffusion solve whose scratch is a static
device array of the library. Called through the C ABI (ctypes) and compared with
getm_tracer_vdiff on the same inputs, two calls in a row, so that the second call runs on scratch
left over from the first. The file is named to be collected last; every test sets up its own
inputs and passes alone in a fresh process as well.

Tolerance: both entry points run the same FP64 kernel, so the results must agree to 1e-13
relative (0 expected)."""
import ctypes as C

import numpy as np
import pytest

from code_b200 import cases
from code_b200 import getm
from code_b200.grid import Grid

from helpers import dev, host, make_ctx

GETM_ERR_ARG = -1
GETM_ERR_TOO_LARGE = -8
MAX_CELLS = 4194304  # GETM_VDIFF_NOALLOC_MAX_CELLS
TOL = 1e-13


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _noalloc(grid, stream, dt, cnpar, avmol, S, hn, nuh, az, src=None):
    dom = grid.domain()
    return getm.lib().getm_tracer_vdiff_noalloc(C.byref(dom), C.c_void_p(stream), dt, cnpar, avmol, _p(S),
                                                _p(hn), _p(nuh), _p(az), _p(src))


def _close(a, b):
    scale = max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max()) <= TOL * scale


def test_too_large_domain_is_rejected():
    """A domain beyond the fixed scratch returns GETM_ERR_TOO_LARGE before any device work (the
    size check comes first, so this runs without a GPU)."""
    g = Grid(300, 300, 50, 100.0, 100.0)
    assert g.ni * g.nj * (g.kmax + 1) > MAX_CELLS
    dom = g.domain()
    fake = C.c_void_p(256)  # never dereferenced: the call returns before using it
    rc = getm.lib().getm_tracer_vdiff_noalloc(C.byref(dom), None, 60.0, 0.9, 1e-9, fake, fake, fake, fake, None)
    assert rc == GETM_ERR_TOO_LARGE


def test_bad_arguments_are_rejected():
    g = Grid(8, 8, 4, 100.0, 100.0)
    dom = g.domain()
    fake = C.c_void_p(256)
    L = getm.lib()
    assert L.getm_tracer_vdiff_noalloc(None, None, 60.0, 0.9, 1e-9, fake, fake, fake, fake, None) == GETM_ERR_ARG
    assert L.getm_tracer_vdiff_noalloc(C.byref(dom), None, 60.0, 0.9, 1e-9, None, fake, fake, fake,
                                       None) == GETM_ERR_ARG


def test_huge_strides_do_not_overflow_the_size_check():
    """Strides so large that sk*(kmax+1) or sj*nj would overflow a 64-bit integer are refused
    (GETM_ERR_TOO_LARGE for the 3D extent, GETM_ERR_ARG for inconsistent strides) before any device
    work: the sizes are compared by division."""
    g = Grid(8, 8, 50, 100.0, 100.0)
    fake = C.c_void_p(256)
    L = getm.lib()
    dom = g.domain()
    dom.sk = 1 << 62  # sk * 51 wraps around in int64
    assert L.getm_tracer_vdiff_noalloc(C.byref(dom), None, 60.0, 0.9, 1e-9, fake, fake, fake, fake,
                                       None) == GETM_ERR_TOO_LARGE
    dom = g.domain()
    dom.sj = 1 << 61  # sj * nj wraps around; sk smaller than sj
    assert L.getm_tracer_vdiff_noalloc(C.byref(dom), None, 60.0, 0.9, 1e-9, fake, fake, fake, fake,
                                       None) == GETM_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("with_src", [False, True])
def test_noalloc_matches_context_entry_two_calls(with_src):
    import torch

    c = cases.random_case(nx=61, ny=47, kmax=23, seed=17)
    g = c.grid
    assert g.ni * g.nj * (g.kmax + 1) <= MAX_CELLS
    dt = c.par["dt"]
    cnpar = float(np.float32(0.9))
    avmol = 1.1e-9
    ctx, m = make_ctx(c)
    az = m[0]
    hn, nuh = dev(c["hn"]), dev(c["nuh"])
    rng = np.random.default_rng(5)
    src = dev(rng.normal(size=c["f"].shape) * 1e-3) if with_src else None
    S_ctx = dev(c["f"])
    S_na = dev(c["f"])
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        ctx.tracer_vdiff(dt, cnpar, avmol, S_ctx, hn, nuh, az, src)
        rc = _noalloc(g, stream, dt, cnpar, avmol, S_na, hn, nuh, az, src)
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        a, b = host(S_na), host(S_ctx)
        assert np.isfinite(a).all()
        assert _close(a, b), f"call {call}: max diff {np.abs(a - b).max()}"
    # the solve changed the field (the comparison is not of two untouched copies)
    assert not np.array_equal(host(S_na), c["f"])
    ctx.close()


@pytest.mark.gpu
def test_noalloc_second_domain_reuses_scratch():
    """Two domains of different shape one after the other on the same scratch."""
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    for nx, ny, kmax, seed in ((33, 70, 12, 2), (90, 40, 30, 4)):
        c = cases.random_case(nx=nx, ny=ny, kmax=kmax, seed=seed)
        ctx, m = make_ctx(c)
        hn, nuh = dev(c["hn"]), dev(c["nuh"])
        S_ctx, S_na = dev(c["f"]), dev(c["f"])
        ctx.tracer_vdiff(c.par["dt"], 0.5, 1.4e-7, S_ctx, hn, nuh, m[0], None)
        assert _noalloc(c.grid, stream, c.par["dt"], 0.5, 1.4e-7, S_na, hn, nuh, m[0]) == 0
        torch.cuda.synchronize()
        assert _close(host(S_na), host(S_ctx))
        ctx.close()
