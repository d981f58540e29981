"""NaN/Inf guard (b200bssn_check_finite): reports the smallest element index with a
non-finite value among the plan's interior points, ignores ghost points."""
import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _setup(ctx):
    import torch

    from test_gpu_parity import BATCH, _fake_batch

    u, blocks, total = _fake_batch(BATCH, seed=2)
    plan = sg.Plan(ctx, blocks, sg.FP64, 6000)
    return plan, blocks, torch.from_numpy(u).cuda(), total


def _elem(b, i, j, k):
    return b.offset + i + b.sz[0] * (j + b.sz[1] * k)


def test_guard_finite_and_planted(ctx):
    plan, blocks, ud, total = _setup(ctx)
    assert plan.check_finite(list(ud)) is None
    b = blocks[4]
    e_nan = _elem(b, 10, 3, 20)
    ud[5, e_nan] = float("nan")
    assert plan.check_finite(list(ud)) == e_nan
    assert plan.check_finite([ud[0]]) is None  # only the arrays asked for are scanned
    b1 = blocks[1]
    e_inf = _elem(b1, 3, 4, 5)
    ud[20, e_inf] = float("-inf")
    assert plan.check_finite(list(ud)) == min(e_nan, e_inf)
    plan.close()


def test_guard_ignores_ghosts(ctx):
    plan, blocks, ud, total = _setup(ctx)
    mask = po.interior_elements(blocks, total)
    inside = np.zeros(total, dtype=bool)
    for b in blocks:
        inside[b.offset:b.offset + b.npad] = True
    import torch

    ghosts = torch.from_numpy(np.nonzero(inside & ~mask)[0]).cuda()
    ud[:, ghosts] = float("nan")
    assert plan.check_finite(list(ud)) is None
    plan.close()


def test_guard_stops_a_blown_up_evolution(ctx):
    """A state that goes non-finite during RK4 steps is caught between steps."""
    plan, blocks, ud, total = _setup(ctx)
    rk = sg.RK4(plan)
    cols = list(ud)
    rk.init(cols)
    prm = sg.Params.make(ko_sigma=0.1)
    b = blocks[0]
    ud[1, _elem(b, 6, 6, 6)] = float("nan")  # chi: spreads through the stencils
    rk.step(cols, 1e-3, prm)
    bad = plan.check_finite(cols)
    assert bad is not None and b.offset <= bad < b.offset + b.npad
    rk.close()
    plan.close()


def test_guard_argument_errors(ctx):
    plan, blocks, ud, total = _setup(ctx)
    import ctypes

    lib = sg.load()
    rc = lib.b200bssn_check_finite(plan.handle, None, 0, None, None)
    assert rc == -1
    plan.close()
