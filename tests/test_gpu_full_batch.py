"""GPU checks on the benchmark's full workload -- the 3000-block two-puncture batch
(1.065e8 interior points, 26.7 GB per state) -- through properties that do not depend
on its size, so the whole batch can be checked where the oracle could only afford a
sample of it:

* chunk invariance: FP64 plans with different chunk sizes (different chunk
  boundaries, scratch reuse and kernel pipelining) give the same bits everywhere;
* the metric's bar: MIXED against FP64 over the whole batch, per variable,
  max|mixed - fp64| / max|fp64| <= 1e-6;
* one block of every size class, evaluated alone through the drop-in on host
  arrays, gives the batch plan's bits for that block; the 13^3 and 21^3 ones are
  also checked against the oracle (FP64 <= 1e-12).
"""
import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po
from sympygr_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-6
SIGMA = 0.4


@pytest.fixture(scope="module")
def batch():
    import torch

    u, blocks = wl.two_puncture_batch_torch(wl.BATCH_SIZES, wl.BATCH_COUNTS, seed=0, device="cuda")
    yield u, blocks
    del u
    torch.cuda.empty_cache()


def _eval(ctx, u, blocks, precision, chunk_points=0):
    import torch

    plan = sg.Plan(ctx, blocks, precision, chunk_points)
    rd = torch.zeros_like(u)
    plan.rhs_device(list(rd), list(u), sg.Params.make(ko_sigma=SIGMA, precision=precision))
    torch.cuda.synchronize()
    nchunks = plan.launches // 3
    plan.close()
    return rd, nchunks


def test_full_batch_properties(ctx, oracle_lib, batch):
    import torch

    u, blocks = batch
    ref, n1 = _eval(ctx, u, blocks, sg.FP64)
    other, n2 = _eval(ctx, u, blocks, sg.FP64, chunk_points=3_000_000)
    assert n1 != n2  # the two plans cut the batch differently
    assert torch.equal(ref, other)
    del other

    mixed, _ = _eval(ctx, u, blocks, sg.MIXED)
    scale = ref.abs().amax(dim=1)
    err = (mixed - ref).abs().amax(dim=1) / torch.clamp(scale, min=1e-300)
    err[scale == 0] = 0
    assert err.max().item() < TOL_MIXED, err.cpu().numpy()
    del mixed

    # one block per class through the drop-in, on host copies of that block alone
    prm = sg.Params.make(ko_sigma=SIGMA)
    for n in wl.BATCH_SIZES:
        b = next(bb for bb in blocks if bb.sz[0] == n)
        ub = np.ascontiguousarray(u[:, b.offset:b.offset + b.npad].cpu().numpy())
        local = wl.Block(0, b.sz, b.bflag, b.pmin, b.pmax)
        rhs = np.zeros_like(ub)
        ctx.bssnrhs(list(rhs), list(ub), 0, local.pmin, local.pmax, local.sz, local.bflag, prm)
        got = po.interior(rhs, local)
        batch_vals = po.interior(ref[:, b.offset:b.offset + b.npad].cpu().numpy(), local)
        assert np.array_equal(got, batch_vals), n
        if n <= 21:
            oracle = po.interior(po.oracle_rhs(ub, local, po.params(ko_sigma=SIGMA)), local)
            mx, _ = po.rel_errors(got, oracle)
            assert mx.max() < TOL64, (n, mx.max())
