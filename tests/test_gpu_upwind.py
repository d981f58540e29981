"""GPU, opt-in upwind mode (plan option `advective`): the advective terms beta^i d_i use
the 4th-order upwind derivatives deriv42adv_* (bssn/src/derivs.cpp:495-900) instead of
the centred 6th-order ones.  Against the oracle's upwind-mode RHS (its upwind operator
is pinned bit for bit to the reference's deriv42adv_* in the CPU tests).

FP64 bar: per variable, max|gpu - oracle| / max|oracle| <= 1e-12 on every block.  MIXED
bar: the same norm over the batch's blocks <= 1e-6, and <= 2e-5 on every block.
"""
import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-6
TOL_MIXED_BLOCK = 2e-5
SIGMA = 0.25


def _batch(seed=7):
    from test_gpu_parity import BATCH, _fake_batch

    return _fake_batch(BATCH, seed=seed)


def _gpu_rhs(ctx, u, blocks, precision, advective, chunk_points=0):
    import torch

    plan = sg.Plan(ctx, blocks, precision, chunk_points, advective=advective)
    ud = torch.from_numpy(u).cuda()
    rd = torch.zeros_like(ud)
    plan.rhs_device(list(rd), list(ud), sg.Params.make(ko_sigma=SIGMA, precision=precision))
    torch.cuda.synchronize()
    plan.close()
    return rd.cpu().numpy()


@pytest.mark.parametrize("chunk_points", [0, 7000])
def test_upwind_fp64_vs_oracle(ctx, oracle_lib, chunk_points):
    u, blocks, total = _batch()
    got = _gpu_rhs(ctx, u, blocks, sg.FP64, True, chunk_points)
    for b in blocks:
        ref = po.interior(po.oracle_rhs_adv(u, b, po.params(ko_sigma=SIGMA)), b)
        mx, _ = po.rel_errors(po.interior(got, b), ref)
        assert mx.max() < TOL64, (b, mx.max(), int(np.argmax(mx)))


def test_upwind_mixed_vs_oracle(ctx, oracle_lib):
    u, blocks, total = _batch(seed=3)
    got = _gpu_rhs(ctx, u, blocks, sg.MIXED, True)
    pairs = [(po.interior(got, b), po.interior(po.oracle_rhs_adv(u, b, po.params(ko_sigma=SIGMA)), b))
             for b in blocks]
    over, per_block = po.batch_rel_errors(pairs)
    assert over.max() < TOL_MIXED, over
    for b, e in zip(blocks, per_block):
        assert e.max() < TOL_MIXED_BLOCK, (b, e.max())


def test_upwind_differs_from_centred_only_through_the_shift(ctx):
    u, blocks, total = _batch(seed=5)
    a = _gpu_rhs(ctx, u, blocks, sg.FP64, False)
    b = _gpu_rhs(ctx, u, blocks, sg.FP64, True)
    m = po.interior_elements(blocks, total)
    assert not np.allclose(a[:, m], b[:, m])
    u0 = u.copy()
    u0[6:9] = 0.0  # no shift: no advection in either mode
    a = _gpu_rhs(ctx, u0, blocks, sg.FP64, False)
    b = _gpu_rhs(ctx, u0, blocks, sg.FP64, True)
    mx, _ = po.rel_errors(b[:, m], a[:, m])
    assert mx.max() < 1e-13


def test_upwind_rk4_vs_oracle(ctx, oracle_lib):
    import torch

    u, blocks, total = _batch(seed=9)
    dt = 2e-3
    ref = u.copy()
    orc = po.OracleRK4(blocks, total, po.params(ko_sigma=SIGMA), advective=True)
    orc.init(ref)
    for _ in range(2):
        orc.step(ref, dt)
    plan = sg.Plan(ctx, blocks, sg.FP64, advective=True)
    rk = sg.RK4(plan)
    ud = torch.from_numpy(u).cuda()
    rk.init(list(ud))
    rk.capture(list(ud), dt, sg.Params.make(ko_sigma=SIGMA), 2)
    rk.launch()
    torch.cuda.synchronize()
    got = ud.cpu().numpy()
    rk.close()
    plan.close()
    m = orc.mask
    mx, _ = po.rel_errors(got[:, m], ref[:, m])
    assert mx.max() < TOL64, mx.max()
