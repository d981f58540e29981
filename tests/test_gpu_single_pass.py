"""GPU: the one-pass MIXED kernel (one persistent launch per evaluation, derivative
scratch in an L2-sized ring of tile-slab slots) against the oracle and against the
two-pass kernels, with rings small enough that items wait for free slots.

MIXED bar: per variable, max|gpu - oracle| / max|oracle| <= 1e-6 over the blocks.
"""
import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-6
SIGMA = 0.3


def _batch():
    from test_gpu_parity import BATCH, _fake_batch

    return _fake_batch(BATCH + [(45, 0x00), (40, 0x30)], seed=13)


def _eval(ctx, u, blocks, **plan_kw):
    import torch

    plan_kw.setdefault("single_pass", True)
    plan = sg.Plan(ctx, blocks, sg.MIXED, **plan_kw)
    ud = torch.from_numpy(u).cuda()
    rd = torch.zeros_like(ud)
    plan.rhs_device(list(rd), list(ud), sg.Params.make(ko_sigma=SIGMA, precision=sg.MIXED))
    plan.status()
    single = plan.single_pass
    plan.close()
    return rd.cpu().numpy(), single


def test_single_pass_only_where_supported(ctx):
    u, blocks, _ = _batch()
    _, single = _eval(ctx, u, blocks)
    assert single
    _, single = _eval(ctx, u, blocks, single_pass=False)
    assert not single
    for kw in ({"precision": sg.FP64}, {"precision": sg.MIXED, "advective": True}):
        plan = sg.Plan(ctx, blocks, single_pass=True, **kw)
        assert not plan.single_pass and plan.launches >= 3
        plan.close()


def test_single_pass_vs_oracle_and_two_pass(ctx, oracle_lib):
    u, blocks, _ = _batch()
    got, _ = _eval(ctx, u, blocks)
    two, _ = _eval(ctx, u, blocks, single_pass=False)
    dmax, rmax = np.zeros(24), np.zeros(24)
    for b in blocks:
        ref = po.interior(po.oracle_rhs(u, b, po.params(ko_sigma=SIGMA)), b)
        g = po.interior(got, b)
        dmax = np.maximum(dmax, np.abs(g - ref).max(axis=1))
        rmax = np.maximum(rmax, np.abs(ref).max(axis=1))
        # the same split-precision derivatives and FP32 algebra as the two-pass kernels
        mx, _ = po.rel_errors(g, po.interior(two, b))
        assert mx.max() < 1e-6, (b.sz, mx.max())
    err = dmax / np.maximum(rmax, 1e-300)
    assert err.max() < TOL_MIXED, err


@pytest.mark.parametrize("ring", [1, 2, 5])
def test_small_rings_give_the_same_bits(ctx, ring):
    """With a ring of 1, 2 or 5 slots every item of a tile-slab waits for the algebra of
    the tile-slab that held its slot before; the values do not depend on the schedule."""
    u, blocks, _ = _batch()
    ref, _ = _eval(ctx, u, blocks)
    got, _ = _eval(ctx, u, blocks, ring_slots=ring)
    assert np.array_equal(got, ref)


def test_single_pass_repeated_evaluations_are_bitwise_stable(ctx):
    import torch

    u, blocks, _ = _batch()
    plan = sg.Plan(ctx, blocks, sg.MIXED, single_pass=True)
    ud = torch.from_numpy(u).cuda()
    prm = sg.Params.make(ko_sigma=SIGMA, precision=sg.MIXED)
    outs = []
    for _ in range(3):
        rd = torch.zeros_like(ud)
        plan.rhs_device(list(rd), list(ud), prm)
        outs.append(rd)
    plan.status()
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    plan.close()
