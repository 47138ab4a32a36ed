"""CPU-side checks of the drop-in boundary: the library loads and exports every entry point that
include/getm_b200.h declares (no compute call needs a GPU), and the Python layer declares the same
set."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "getm_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(getm_[a-z0-9_]+)\s*\(", txt)))


def test_header_parses():
    syms = header_symbols()
    assert "getm_do_advection_3d" in syms and "getm_tracer_vdiff" in syms
    assert len(syms) >= 20


def test_library_exports_header_symbols():
    from code_b200 import build as cb

    lib_path = cb.build()
    lib = ctypes.CDLL(lib_path)
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_layer_declares_all():
    from code_b200 import getm

    declared = set(getm.exported_symbols())
    assert set(header_symbols()) <= declared | {"getm_adv_split_u", "getm_adv_split_v"}, \
        sorted(set(header_symbols()) - declared)


def test_context_requires_cuda():
    import torch

    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from code_b200.getm import Context
    from code_b200.grid import Grid

    with pytest.raises(RuntimeError):
        Context(Grid(8, 8, 4, 100.0, 100.0))


def test_version_string():
    from code_b200 import getm

    assert b"sm_100a" in getm.lib().getm_version()


def test_state_struct_matches_header():
    """The Python mirror of getm_bc_state and the field / parameter name lists have the sizes that
    include/getm_b200.h declares (GETM_NF2, GETM_NF3, GETM_NPD, GETM_NPI)."""
    from code_b200 import state as S
    from code_b200.getm import BcState

    txt = open(os.path.join(ROOT, "include", "getm_b200.h")).read()
    n = {k: int(v) for k, v in re.findall(r"#define GETM_(NF2|NF3|NPD|NPI) (\d+)", txt)}
    assert n == {"NF2": len(S.F2_NAMES), "NF3": len(S.F3_NAMES), "NPD": len(S.PD_NAMES), "NPI": len(S.PI_NAMES)}
    f = dict((name, t) for name, t in BcState._fields_)
    assert (f["f2"]._length_, f["f3"]._length_, f["par"]._length_, f["ipar"]._length_) == (
        n["NF2"], n["NF3"], n["NPD"], n["NPI"])
