"""GPU parity of the Hamiltonian and momentum constraints: the CUDA path through the C
ABI (b200bssn_physical_constraints, b200bssn_constraints_plan_device) against the
reference's own physical_constraints (golden fixtures) and the oracle.

FP64 bar: per constraint, max|gpu - ref| / max|ref| <= 1e-12 over the interior.
MIXED bar (split-precision stencils, FP32 algebra): the same norm <= 1e-6.
"""
import os

import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po
from sympygr_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-6


def _gpu_con(ctx, u, blk, precision=sg.FP64, sentinel=np.nan):
    con = np.full((4, u.shape[1]), sentinel)
    ctx.physical_constraints(list(con), list(u), blk.offset, blk.pmin, blk.pmax, blk.sz, blk.bflag,
                             precision)
    return con


@pytest.mark.parametrize("case", ["con_fake_13_b00", "con_fake_17_b2a"])
def test_dropin_constraints_vs_reference_golden(ctx, golden_dir, case):
    g = np.load(os.path.join(golden_dir, case + ".npz"))
    u, blk = po.fake_block(int(g["n"]), tuple(g["pmin"]), float(g["h"]), int(g["bflag"]))
    con = _gpu_con(ctx, u, blk)
    mx, _ = po.rel_errors(po.interior(con, blk), g["con_interior"])
    assert mx.max() < TOL64, mx
    mask = ~wl.interior_mask(blk).ravel()
    assert np.isnan(con[:, mask]).all()  # ghosts untouched


def test_dropin_constraints_bl_vs_reference_golden(ctx, golden_dir):
    g = np.load(os.path.join(golden_dir, "con_bl_70.npz"))
    u, blk = wl.brill_lindquist(70, 8.0, 1.0)
    c = po.interior(_gpu_con(ctx, u, blk), blk)
    scale = np.maximum(g["checksums"][:, 2], 1e-300)[:, None]
    assert (np.abs(c[:, g["sample_index"]] - g["sample_con"]) / scale).max() < TOL64
    assert np.all(c[1:] == 0.0)


@pytest.mark.parametrize("n,bflag", [(13, 0x3F), (21, 0x15), (30, 0x2A)])
def test_dropin_constraints_vs_oracle(ctx, oracle_lib, n, bflag):
    u, blk = po.fake_block(n, (-0.45, 0.2, -0.3), 0.9 / n, bflag)
    ref = po.interior(po.oracle_constraints(u, blk), blk)
    got = po.interior(_gpu_con(ctx, u, blk), blk)
    mx, _ = po.rel_errors(got, ref)
    assert mx.max() < TOL64, mx
    got32 = po.interior(_gpu_con(ctx, u, blk, sg.MIXED), blk)
    mx32, _ = po.rel_errors(got32, ref)
    assert mx32.max() < TOL_MIXED, mx32


def _fake_batch(seed=7):
    from test_gpu_parity import BATCH, _fake_batch as fb

    return fb(BATCH, seed=seed)


@pytest.mark.parametrize("chunk_points", [0, 4000])
def test_plan_constraints_and_norms_vs_oracle(ctx, oracle_lib, chunk_points):
    import torch

    u, blocks, total = _fake_batch()
    plan = sg.Plan(ctx, blocks, sg.FP64, chunk_points)
    ud = torch.from_numpy(u).cuda()
    cd = torch.full((4, total), float("nan"), dtype=torch.float64, device="cuda")
    norms = torch.full((len(blocks) * 8,), 123.0, dtype=torch.float64, device="cuda")
    plan.constraints_device(list(ud), list(cd), norms)
    torch.cuda.synchronize()
    got = cd.cpu().numpy()
    nrm = norms.cpu().numpy().reshape(len(blocks), 8)
    for bi, b in enumerate(blocks):
        ref = po.interior(po.oracle_constraints(u, b), b)
        gi = po.interior(got, b)
        mx, _ = po.rel_errors(gi, ref)
        assert mx.max() < TOL64, (b, mx)
        assert np.allclose(nrm[bi, :4], (gi ** 2).sum(axis=1), rtol=1e-12, atol=0)
        assert np.array_equal(nrm[bi, 4:], np.abs(gi).max(axis=1))
    plan.close()


def test_plan_constraints_norms_only_and_nan_detection(ctx):
    import torch

    u, blocks, total = _fake_batch(seed=3)
    plan = sg.Plan(ctx, blocks, sg.FP64, 5000)
    ud = torch.from_numpy(u).cuda()
    ref = torch.zeros(len(blocks) * 8, dtype=torch.float64, device="cuda")
    cd = [torch.zeros(total, dtype=torch.float64, device="cuda") for _ in range(4)]
    plan.constraints_device(list(ud), cd, ref)
    norms = torch.zeros_like(ref)
    plan.constraints_device(list(ud), None, norms)  # norms only: same numbers
    torch.cuda.synchronize()
    assert torch.allclose(norms, ref, rtol=1e-13, atol=0)
    # a NaN in the state at an interior point of block 2 shows up as NaN maxima there
    b = blocks[2]
    pp = b.offset + 5 + b.sz[0] * (5 + b.sz[1] * 5)
    ud[1, pp] = float("nan")  # chi
    plan.constraints_device(list(ud), None, norms)
    torch.cuda.synchronize()
    nrm = norms.cpu().numpy().reshape(len(blocks), 8)
    assert np.isnan(nrm[2, 4])
    others = np.delete(nrm, 2, axis=0)
    assert np.isfinite(others).all()
    plan.close()


def test_constraints_errors_are_reported(ctx):
    import torch

    u, blk = po.fake_block(13, (0.0, 0.0, 0.0), 0.1, 0)
    plan = sg.Plan(ctx, [blk], sg.FP64)
    ud = torch.from_numpy(u).cuda()
    with pytest.raises(sg.B200BssnError) as ei:
        plan.constraints_device(list(ud), None, None)
    assert ei.value.code == -1
    plan.close()
