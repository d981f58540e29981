"""GPU parity: the CUDA path through the C ABI against the oracle (C restatement of
the reference's bssnrhs) and the reference's own outputs (golden fixtures).

FP64 bar: per variable, max|gpu - ref| / max|ref| <= 1e-12 over the interior.
MIXED bar (FP32 algebra): the same norm-wise error <= 1e-6 per variable (the benchmark's bar).
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


def _gpu_block(ctx, u, blk, sigma, precision=sg.FP64, sentinel=np.nan):
    rhs = np.full_like(u, sentinel)
    prm = sg.Params.make(ko_sigma=sigma, precision=precision)
    ctx.bssnrhs(list(rhs), list(u), blk.offset, blk.pmin, blk.pmax, blk.sz, blk.bflag, prm)
    return rhs


@pytest.mark.parametrize("case", ["fake_13_b00", "fake_13_b3f", "fake_13_b05", "fake_17_b2a"])
def test_dropin_vs_reference_golden(ctx, golden_dir, case):
    g = np.load(os.path.join(golden_dir, case + ".npz"))
    u, blk = po.fake_block(int(g["n"]), tuple(g["pmin"]), float(g["h"]), int(g["bflag"]))
    rhs = _gpu_block(ctx, u, blk, float(g["sigma"]))
    mx, _ = po.rel_errors(po.interior(rhs, blk), g["rhs_interior"])
    assert mx.max() < TOL64, (mx.max(), int(np.argmax(mx)))
    # ghost points keep the caller's values (the reference leaves them untouched)
    mask = ~wl.interior_mask(blk).ravel()
    assert np.isnan(rhs[:, mask]).all()


@pytest.mark.parametrize("n,bflag", [(13, 0x00), (14, 0x3F), (21, 0x15), (29, 0x2A), (38, 0x01),
                                     (45, 0x30), (37, 0x0C)])
def test_dropin_vs_oracle_fake(ctx, oracle_lib, n, bflag):
    u, blk = po.fake_block(n, (-0.45, 0.2, -0.3), 0.9 / n, bflag)
    prm = po.params(ko_sigma=0.25)
    ref = po.interior(po.oracle_rhs(u, blk, prm), blk)
    got = po.interior(_gpu_block(ctx, u, blk, 0.25), blk)
    mx, _ = po.rel_errors(got, ref)
    assert mx.max() < TOL64, (mx.max(), int(np.argmax(mx)))


def test_dropin_offsets_and_staging_reuse(ctx, oracle_lib):
    """Three blocks zipped into one set of arrays, evaluated one by one through the
    drop-in in an order that grows the context's staging buffers and then reuses them
    for a smaller block (the 70^3 block's 66 MB are staged by several host threads):
    each call writes its block's interior and nothing else."""
    sizes, flags = (21, 70, 45), (0x15, 0x00, 0x2A)
    offsets = np.cumsum((0,) + tuple(n ** 3 for n in sizes))
    u = np.zeros((24, int(offsets[-1])))
    blocks = []
    for n, bf, off in zip(sizes, flags, offsets):
        ub, b = po.fake_block(n, (-0.4, 0.1, -0.2), 1.1 / n, bf)
        u[:, off:off + n ** 3] = ub
        blocks.append(wl.Block(int(off), b.sz, bf, b.pmin, b.pmax))
    rhs = np.full_like(u, np.nan)
    prm = sg.Params.make(ko_sigma=0.3)
    written = np.zeros(u.shape[1], dtype=bool)
    for b in (blocks[0], blocks[1], blocks[2]):
        ctx.bssnrhs(list(rhs), list(u), b.offset, b.pmin, b.pmax, b.sz, b.bflag, prm)
        written[b.offset:b.offset + b.npad] |= wl.interior_mask(b).ravel()
        assert np.isnan(rhs[:, ~written]).all()
        assert not np.isnan(rhs[:, written]).any()
    for b in blocks:
        ref = po.interior(po.oracle_rhs(u, b, po.params(ko_sigma=0.3)), b)
        mx, _ = po.rel_errors(po.interior(rhs, b), ref)
        assert mx.max() < TOL64, (b.sz, mx.max())


def test_cfg1_sines_vs_golden(ctx, golden_dir):
    g = np.load(os.path.join(golden_dir, "sines_38.npz"))
    u, blk = wl.flat_sines(38, 0.1, 0)
    got = po.interior(_gpu_block(ctx, u, blk, float(g["sigma"])), blk)
    scale = g["checksums"][:, 2][:, None]
    err = np.abs(got[:, g["sample_index"]] - g["sample_rhs"]) / scale
    assert err.max() < TOL64
    assert np.allclose(np.abs(got).max(axis=1), g["checksums"][:, 2], rtol=1e-11, atol=0)


def test_cfg2_brill_lindquist_vs_golden_and_oracle(ctx, golden_dir, oracle_lib):
    g = np.load(os.path.join(golden_dir, "bl_134.npz"))
    u, blk = wl.brill_lindquist(134, 8.0, 1.0)
    got = po.interior(_gpu_block(ctx, u, blk, float(g["sigma"])), blk)
    scale = g["checksums"][:, 2][:, None]
    err = np.abs(got[:, g["sample_index"]] - g["sample_rhs"]) / np.maximum(scale, 1e-300)
    assert err.max() < TOL64
    ref = po.interior(po.oracle_rhs(u, blk, po.params(ko_sigma=float(g["sigma"]))), blk)
    mx, _ = po.rel_errors(got, ref)
    # variables whose RHS is identically zero here have ref max 0: compare absolutely
    zero = np.abs(ref).max(axis=1) == 0
    assert mx[~zero].max() < TOL64
    assert np.abs(got[zero]).max() < 1e-300 if zero.any() else True


def _fake_batch(sizes_flags, seed=7):
    """Block list of fake_initial_data blocks at scattered offsets."""
    rng = np.random.default_rng(seed)
    blocks, off = [], 0
    for n, bflag in sizes_flags:
        h = float(rng.uniform(0.02, 0.08))
        pmin = tuple(float(t) for t in rng.uniform(-1.0, 0.5, 3))
        off += int(rng.integers(0, 40))
        blocks.append(wl.Block(off, (n, n, n), bflag, pmin, tuple(pmin[a] + (n - 1) * h for a in range(3))))
        off += n ** 3
    u = np.zeros((24, off))
    for b in blocks:
        x, y, z = wl.coords(b)
        u[:, b.offset:b.offset + b.npad] = po.fake_initial_data(x, y, z).reshape(24, -1)
    return u, blocks, off


BATCH = [(13, 0), (13, 0x3F), (21, 0x04), (16, 0x21), (37, 0), (13, 0x12), (25, 0x08)]


@pytest.mark.parametrize("chunk_points", [0, 9000])
def test_batch_device_vs_oracle(ctx, oracle_lib, chunk_points):
    import torch

    u, blocks, total = _fake_batch(BATCH)
    plan = sg.Plan(ctx, blocks, sg.FP64, chunk_points)
    assert plan.points == sum(b.ninterior for b in blocks)
    ud = torch.from_numpy(u).cuda()
    rd = torch.zeros_like(ud)
    prm = sg.Params.make(ko_sigma=0.15)
    plan.rhs_device(list(rd), list(ud), prm)
    torch.cuda.synchronize()
    got = rd.cpu().numpy()
    for b in blocks:
        ref = po.oracle_rhs(u, b, po.params(ko_sigma=0.15))
        mx, _ = po.rel_errors(po.interior(got, b), po.interior(ref, b))
        assert mx.max() < TOL64, (b, mx.max())
    plan.close()


def test_chunking_is_bitwise_invariant(ctx):
    import torch

    u, blocks, total = _fake_batch(BATCH, seed=11)
    ud = torch.from_numpy(u).cuda()
    prm = sg.Params.make(ko_sigma=0.2)
    outs = []
    for cp in (0, 5000, 20000):
        plan = sg.Plan(ctx, blocks, sg.FP64, cp)
        rd = torch.zeros_like(ud)
        plan.rhs_device(list(rd), list(ud), prm)
        torch.cuda.synchronize()
        outs.append(rd.cpu())
        plan.close()
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])


@pytest.mark.parametrize("chunk_points", [0, 3000])  # 3000: several chunks, pipelined copies
@pytest.mark.parametrize("policy", [sg.GHOSTS_PRESERVE, sg.GHOSTS_ZERO])
def test_batch_host_ghost_policy(ctx, oracle_lib, policy, chunk_points):
    # small blocks and two whose interiors come back as strided boxes under PRESERVE
    u, blocks, total = _fake_batch(BATCH[:4] + [(37, 0x00), (45, 0x2A)], seed=5)
    plan = sg.Plan(ctx, blocks, sg.FP64, chunk_points)
    assert chunk_points == 0 or plan.launches >= 6
    rhs = np.full_like(u, 7.0)
    prm = sg.Params.make(ko_sigma=0.1, ghost_policy=policy)
    plan.rhs_host(list(rhs), list(u), total, prm)
    for b in blocks:
        ref = po.oracle_rhs(u, b, po.params(ko_sigma=0.1))
        mx, _ = po.rel_errors(po.interior(rhs, b), po.interior(ref, b))
        assert mx.max() < TOL64
        seg = rhs[:, b.offset:b.offset + b.npad]
        ghosts = seg[:, ~wl.interior_mask(b).ravel()]
        assert np.all(ghosts == (7.0 if policy == sg.GHOSTS_PRESERVE else 0.0))
    # elements between blocks follow the same policy
    inside = np.zeros(total, dtype=bool)
    for b in blocks:
        inside[b.offset:b.offset + b.npad] = True
    lo = min(b.offset for b in blocks)
    gaps = rhs[:, lo:][:, ~inside[lo:]]
    assert np.all(gaps == (7.0 if policy == sg.GHOSTS_PRESERVE else 0.0))
    plan.close()


@pytest.mark.parametrize("chunk_points", [0, 3000])
def test_batch_host_ghost_policy_sequence(ctx, chunk_points):
    """One plan alternating the two policies: a ghost-preserving call puts the caller's
    RHS values into the plan's device staging, so the next zeroing call must clear them
    again; repeated zeroing calls keep zeros; the interiors never change."""
    u, blocks, total = _fake_batch(BATCH[:4] + [(37, 0x00)], seed=9)
    plan = sg.Plan(ctx, blocks, sg.FP64, chunk_points)
    ghost = np.ones(total, dtype=bool)
    for b in blocks:
        ghost[b.offset:b.offset + b.npad] &= ~wl.interior_mask(b).ravel()
    ref = None
    for policy, fill in ((sg.GHOSTS_ZERO, 3.0), (sg.GHOSTS_PRESERVE, 7.0), (sg.GHOSTS_ZERO, 5.0),
                         (sg.GHOSTS_ZERO, 6.0), (sg.GHOSTS_PRESERVE, 8.0)):
        rhs = np.full_like(u, fill)
        plan.rhs_host(list(rhs), list(u), total, sg.Params.make(ko_sigma=0.1, ghost_policy=policy))
        lo = min(b.offset for b in blocks)
        g = rhs[:, lo:][:, ghost[lo:]]
        assert np.all(g == (fill if policy == sg.GHOSTS_PRESERVE else 0.0)), (policy, fill)
        inner = rhs[:, ~ghost]
        if ref is None:
            ref = inner.copy()
        assert np.array_equal(inner, ref)
    plan.close()


@pytest.mark.parametrize("maker", ["fake", "sines", "bl"])
def test_mixed_precision_error(ctx, oracle_lib, maker):
    if maker == "fake":
        u, blk = po.fake_block(29, (-0.45, 0.2, -0.3), 0.03, 0x15)
    elif maker == "sines":
        u, blk = wl.flat_sines(38, 0.1, 0)
    else:
        u, blk = wl.brill_lindquist(70, 8.0, 1.0)
    ref = po.interior(po.oracle_rhs(u, blk, po.params(ko_sigma=0.4)), blk)
    got = po.interior(_gpu_block(ctx, u, blk, 0.4, precision=sg.MIXED), blk)
    mx, rms = po.rel_errors(got, ref)
    nz = np.abs(ref).max(axis=1) > 0
    assert mx[nz].max() < TOL_MIXED, (maker, mx.max(), int(np.argmax(mx)))


def test_two_puncture_batch_mixed_vs_fp64(ctx):
    import torch

    sizes, counts = (13, 21, 37), (20, 8, 3)
    u, blocks = wl.two_puncture_batch_torch(sizes, counts, seed=3, device="cuda")
    outs = {}
    for prec in (sg.FP64, sg.MIXED):
        plan = sg.Plan(ctx, blocks, prec)
        rd = torch.zeros_like(u)
        plan.rhs_device(list(rd), list(u), sg.Params.make(ko_sigma=0.4, precision=prec))
        torch.cuda.synchronize()
        outs[prec] = rd
        plan.close()
    a, b = outs[sg.FP64], outs[sg.MIXED]
    for v in range(24):
        s = a[v].abs().max().item()
        if s > 0:
            assert (a[v] - b[v]).abs().max().item() / s < TOL_MIXED, v


def test_errors_are_reported(ctx):
    u, blk = po.fake_block(13, (0.0, 0.0, 0.0), 0.1, 0)
    bad = wl.Block(0, (12, 13, 13), 0, blk.pmin, blk.pmax)
    with pytest.raises(sg.B200BssnError) as ei:
        sg.Plan(ctx, [bad])
    assert ei.value.code == -2
    plan = sg.Plan(ctx, [blk], sg.FP64)
    import torch

    ud = torch.from_numpy(u).cuda()
    with pytest.raises(sg.B200BssnError) as ei:
        plan.rhs_device(list(ud), list(ud), sg.Params.make(precision=sg.MIXED))
    assert ei.value.code == -1
    plan.close()


@pytest.mark.parametrize("sz,bflag", [((13, 21, 17), 0x00), ((19, 13, 25), 0x3F), ((23, 17, 13), 0x26)])
def test_non_cubic_blocks_vs_oracle(ctx, oracle_lib, sz, bflag):
    """Blocks with different extents and spacings per axis (the reference derives h per
    axis, rhs.cpp:144-146) through the drop-in and through a plan."""
    import torch

    from sympygr_b200 import workloads as wl

    pmin = (-0.37, 0.11, -0.23)
    h = (0.031, 0.027, 0.043)
    blk = wl.Block(5, sz, bflag, pmin, tuple(pmin[a] + (sz[a] - 1) * h[a] for a in range(3)))
    x, y, z = wl.coords(blk)
    u = np.zeros((24, 5 + blk.npad))
    u[:, 5:] = po.fake_initial_data(x, y, z).reshape(24, -1)
    ref = po.interior(po.oracle_rhs(u, blk, po.params(ko_sigma=0.3)), blk)
    got = po.interior(_gpu_block(ctx, u, blk, 0.3), blk)
    mx, _ = po.rel_errors(got, ref)
    assert mx.max() < TOL64, mx.max()
    plan = sg.Plan(ctx, [blk], sg.FP64, 600, slab_depth=4)  # 4-plane slabs over several chunks
    assert plan.launches >= 6
    ud = torch.from_numpy(u).cuda()
    rd = torch.zeros_like(ud)
    plan.rhs_device(list(rd), list(ud), sg.Params.make(ko_sigma=0.3))
    torch.cuda.synchronize()
    mx, _ = po.rel_errors(po.interior(rd.cpu().numpy(), blk), ref)
    assert mx.max() < TOL64, mx.max()
    plan.close()


def test_plan_argument_checks(ctx):
    u, blk = po.fake_block(13, (0.0, 0.0, 0.0), 0.1, 0)
    for bad in ([], [wl.Block(0, (13, 13, 13), 0x40, blk.pmin, blk.pmax)],
                [wl.Block(0, (13, 13, 13), 0, blk.pmax, blk.pmin)]):
        with pytest.raises(sg.B200BssnError) as ei:
            sg.Plan(ctx, bad)
        assert ei.value.code == -1
