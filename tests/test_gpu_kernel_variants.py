"""GPU: the tuning variants of the two-pass derivative kernels (tile height 4, 8, 16;
register splits 96/128, 80/96, 128/168; two output points per thread on 16x16 tiles)
compute the same derivatives with
the same operations in the same order, so every variant must reproduce the default
plan bit for bit, in FP64 and MIXED, on blocks with flagged faces; and the default
FP64 result stays pinned to the oracle."""
import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

VARIANTS = [(4, 1, 1), (16, 1, 1), (8, 1, 1), (8, 2, 1), (8, 3, 1), (16, 0, 2)]  # tile_y, regs, points/thread


def _batch():
    from test_gpu_parity import BATCH, _fake_batch

    return _fake_batch(BATCH + [(40, 0x0F), (23, 0x30)], seed=21)


def _eval(ctx, u, blocks, precision, **kw):
    import torch

    plan = sg.Plan(ctx, blocks, precision, **kw)
    ud = torch.from_numpy(u).cuda()
    rd = torch.zeros_like(ud)
    plan.rhs_device(list(rd), list(ud), sg.Params.make(ko_sigma=0.2, precision=precision))
    torch.cuda.synchronize()
    plan.close()
    return rd.cpu().numpy()


@pytest.mark.parametrize("precision", [sg.FP64, sg.MIXED], ids=["fp64", "mixed"])
def test_variants_reproduce_the_default_bitwise(ctx, oracle_lib, precision):
    u, blocks, _ = _batch()
    ref = _eval(ctx, u, blocks, precision)
    if precision == sg.FP64:
        for b in blocks:
            o = po.interior(po.oracle_rhs(u, b, po.params(ko_sigma=0.2)), b)
            mx, _ = po.rel_errors(po.interior(ref, b), o)
            assert mx.max() < 1e-12, (b, mx.max())
    for ty, regs, ppt in VARIANTS:
        got = _eval(ctx, u, blocks, precision, tile_y=ty, deriv_regs=regs, points_per_thread=ppt, slab_depth=16)
        assert np.array_equal(got, ref), (ty, regs, ppt)


def test_unbuilt_variants_are_refused(ctx):
    u, blocks, _ = _batch()
    for kw in ({"tile_y": 12}, {"tile_y": 4, "deriv_regs": 2}, {"deriv_regs": 4},
               {"advective": True, "tile_y": 16}, {"advective": True, "deriv_regs": 3},
               {"points_per_thread": 2, "tile_y": 8}, {"points_per_thread": 2, "advective": True},
               {"points_per_thread": 3}):
        with pytest.raises(sg.B200BssnError) as ei:
            sg.Plan(ctx, blocks, sg.FP64, **kw)
        assert ei.value.code == -1
