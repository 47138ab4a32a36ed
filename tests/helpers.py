"""Shared helpers of the test suite (numpy <-> device, oracle runs of the same inputs)."""
from __future__ import annotations

import numpy as np


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def rel_err(a, b, floor=1e-30):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(a - b)
    s = np.maximum(np.abs(b), floor)
    return float((d / s).max()) if d.size else 0.0


def max_abs(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max())


def make_ctx(case):
    """GPU context with the case's masks installed; returns (ctx, device masks)."""
    from code_b200.getm import Context

    ctx = Context(case.grid)
    m = [dev(x) for x in case.masks()]
    ctx.init_advection(*m)
    return ctx, m
