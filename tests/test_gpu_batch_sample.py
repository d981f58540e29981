"""GPU parity on the benchmark's own blocks: a class-proportional sample of the
two-puncture batch (the 69^3 and 135^3 classes included, some blocks with flagged
faces) through a multi-chunk plan at the default slab depth (FP64, and MIXED on its two-pass
kernels) and through the one-pass MIXED kernel, against
the oracle (the C restatement of the reference's bssnrhs, pinned to the reference's
outputs by the CPU tests).

Bars, per variable, max|gpu - oracle| / max|oracle|:
FP64 <= 1e-12 on every block.  MIXED <= 1e-6 over the sample's interior points (the
norm the benchmark reports over the whole batch), and <= 2e-5 on every block: on
blocks far from both punctures the K and At right-hand sides are sums of second
derivatives of the lapse and chi that cancel to a few percent of their terms (the
lapse is close to harmonic there), so the 6e-8 rounding of FP32 lifts the error
relative to that block's own largest value to a few 1e-6 (up to 1.1e-5 measured on a
21^3 block with flagged faces).
"""
import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po
from sympygr_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-6
TOL_MIXED_BLOCK = 2e-5
SIGMA = 0.4
# indices into the seed-0 batch: per class some blocks with a face mask and some without
# (135^3: #2970 bflag 0x1f; 69^3: #2860 0x23; 37^3: #2550 0x2c; 21^3: #1808 0x2b; 13^3: #0 0x0c)
SAMPLE = [2970, 2971, 2860, 2861, 2550, 2551, 1808, 1809, 1810, 0, 1, 2, 3]
CHUNK_POINTS = 1_000_000  # several chunks; a 135^3 block's 48-plane slab is 0.8M points


@pytest.fixture(scope="module")
def sample():
    blocks, _ = wl.batch_blocks(seed=0)
    picked = [blocks[i] for i in SAMPLE]
    out, off = [], 0
    for b in picked:
        out.append(wl.Block(off, b.sz, b.bflag, b.pmin, b.pmax))
        off += ((b.npad + 31) // 32) * 32
    u = np.zeros((24, off))
    punct = [(-4.0, 0.0, 0.0, 0.5), (4.0, 0.0, 0.0, 0.5)]
    for b in out:
        x, y, z = wl.coords(b)
        wl._bl_fields(u, slice(b.offset, b.offset + b.npad), x, y, z, punct)
    refs = [po.interior(po.oracle_rhs(u, b, po.params(ko_sigma=SIGMA)), b) for b in out]
    return u, out, refs


def _run(ctx, u, blocks, precision, two_pass):
    import torch

    plan = sg.Plan(ctx, blocks, precision, CHUNK_POINTS, single_pass=not two_pass)
    if plan.single_pass:
        assert plan.launches == 1  # the one-pass kernel over every block
    else:
        assert plan.launches >= 2 * 3  # more than one chunk
    ud = torch.from_numpy(u).cuda()
    rd = torch.zeros_like(ud)
    plan.rhs_device(list(rd), list(ud), sg.Params.make(ko_sigma=SIGMA, precision=precision))
    plan.status()
    plan.close()
    return rd.cpu().numpy()


def test_sample_has_the_large_classes_and_flagged_faces(sample):
    _, blocks, _ = sample
    sizes = {b.sz[0] for b in blocks}
    assert {13, 21, 37, 69, 135} <= sizes
    assert any(b.bflag and b.sz[0] == 135 for b in blocks)
    assert any(b.bflag and b.sz[0] == 69 for b in blocks)


@pytest.mark.parametrize("precision,two_pass,tol_all,tol_block",
                         [(sg.FP64, True, TOL64, TOL64), (sg.MIXED, False, TOL_MIXED, TOL_MIXED_BLOCK),
                          (sg.MIXED, True, TOL_MIXED, TOL_MIXED_BLOCK)],
                         ids=["fp64", "mixed-one-pass", "mixed-two-pass"])
def test_batch_sample_vs_oracle(ctx, oracle_lib, sample, precision, two_pass, tol_all, tol_block):
    u, blocks, refs = sample
    got = _run(ctx, u, blocks, precision, two_pass)
    over, per_block = po.batch_rel_errors([(po.interior(got, b), ref) for b, ref in zip(blocks, refs)])
    for b, e in zip(blocks, per_block):
        print(f"precision={precision} n={b.sz[0]} bflag={b.bflag:#04x} per-block max rel err {e.max():.3e} "
              f"(variable {int(np.argmax(e))})")
    print(f"precision={precision} per-variable max rel err over the sample {over.max():.3e}")
    assert over.max() < tol_all, over
    worst = max(range(len(blocks)), key=lambda k: per_block[k].max())
    assert per_block[worst].max() < tol_block, (blocks[worst].sz, hex(blocks[worst].bflag), per_block[worst])
