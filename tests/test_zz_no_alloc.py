"""The allocation-free entry point b200bssn_rhs_noalloc, called through the C ABI.

It serves callers that cannot call cudaMalloc (a framework whose pool allocator
owns the GPU's memory, or a time-step loop that must not trigger the device-wide
synchronisation of cudaMalloc/cudaFree): its scratch is a fixed device array
inside the library.  Its output must agree with the regular plan-based entry point
(b200bssn_rhs_plan_device) on the same inputs, call after call, although every
call reuses the array the previous call left behind.

Kept in a file that pytest collects last; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po
from sympygr_b200 import capi
from sympygr_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL64 = 1e-12   # same bar as the other FP64 parity tests
TOL_MIXED = 1e-6


def _pair(ctx, u_np, blk, sigma, precision):
    """(noalloc result, regular entry point result) as numpy arrays."""
    import torch

    torch.cuda.set_device(0)
    ud = torch.from_numpy(u_np).cuda()
    r_noalloc = torch.full_like(ud, float("nan"))
    r_regular = torch.full_like(ud, float("nan"))
    prm = sg.Params.make(ko_sigma=sigma, precision=precision)
    stream = torch.cuda.current_stream()
    capi.rhs_noalloc(list(r_noalloc), list(ud), blk, prm, stream=stream.cuda_stream)
    stream.synchronize()
    plan = sg.Plan(ctx, [blk], precision)
    plan.rhs_device(list(r_regular), list(ud), prm)
    torch.cuda.synchronize()
    plan.close()
    return r_noalloc.cpu().numpy(), r_regular.cpu().numpy()


def _check(a, b, blk, tol):
    ia, ib = po.interior(a, blk), po.interior(b, blk)
    assert np.isfinite(ia).all()
    mx, _ = po.rel_errors(ia, ib)
    nz = np.abs(ib).max(axis=1) > 0
    assert mx[nz].max() < tol, mx.max()
    assert np.array_equal(ia[~nz], ib[~nz])
    # ghost points are not written
    mask = ~wl.interior_mask(blk).ravel()
    assert np.isnan(a[:, mask]).all()


def test_noalloc_matches_regular_entry_point_two_calls(ctx):
    # call 1: a 21^3 block with three flagged faces
    u1, b1 = po.fake_block(21, (-0.35, 0.15, -0.2), 0.04, 0x15)
    a, b = _pair(ctx, u1, b1, 0.3, sg.FP64)
    _check(a, b, b1, TOL64)
    # call 2 reuses the same fixed array: a different, larger block (38^3, the cap)
    u2, b2 = wl.flat_sines(38, 0.1, 0)
    a, b = _pair(ctx, u2, b2, 0.4, sg.FP64)
    _check(a, b, b2, TOL64)
    # and back to the first block, now in mixed precision
    a, b = _pair(ctx, u1, b1, 0.3, sg.MIXED)
    _check(a, b, b1, TOL_MIXED)


def test_noalloc_refuses_blocks_over_the_limit(ctx):
    import torch

    n = 40  # 34^3 = 39304 interior points > 32768
    assert (n - 6) ** 3 > capi.NOALLOC_MAX_POINTS
    ud = torch.zeros((24, n ** 3), dtype=torch.float64, device="cuda")
    blk = wl.Block(0, (n, n, n), 0, (0.0,) * 3, (1.0,) * 3)
    with pytest.raises(sg.B200BssnError) as ei:
        capi.rhs_noalloc(list(ud), list(ud), blk, sg.Params.make())
    assert ei.value.code == -8


def _elongated(sz, bflag):
    """A non-cubic fake_initial_data block; its interior spans several 48-plane z-slabs."""
    pmin = (-0.4, 0.1, -0.9)
    h = 0.035
    blk = wl.Block(0, sz, bflag, pmin, tuple(pmin[a] + (sz[a] - 1) * h for a in range(3)))
    x, y, z = wl.coords(blk)
    return po.fake_initial_data(x, y, z).reshape(24, -1).copy(), blk


@pytest.mark.parametrize("precision,tol", [(sg.FP64, TOL64), (sg.MIXED, TOL_MIXED)],
                         ids=["fp64", "mixed"])
@pytest.mark.parametrize("sz,bflag", [((13, 13, 55), 0x00), ((13, 13, 55), 0x30),
                                      ((20, 16, 110), 0x3F)])
def test_noalloc_multi_slab_blocks(ctx, sz, bflag, precision, tol):
    """Blocks whose interior spans several z-slabs: a slab starting at a scratch point
    that is not on a 32-point boundary, runs past a slab's end, and a trailing slab of
    one plane (13x13x55: 49 interior planes = 48 + 1) or eight (20x16x110: 48 + 48 + 8),
    with and without flagged z faces next to the short slab."""
    u, blk = _elongated(sz, bflag)
    assert (blk.sz[0] - 6) * (blk.sz[1] - 6) * (blk.sz[2] - 6) <= capi.NOALLOC_MAX_POINTS
    a, b = _pair(ctx, u, blk, 0.3, precision)
    _check(a, b, blk, tol)
