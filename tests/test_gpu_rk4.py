"""GPU RK4 time stepping (b200bssn_rk4_*) against the oracle's RK4 (the oracle's
right-hand side inside classic RK4, oracle/pyoracle.py OracleRK4).

FP64 bar: per variable, max|gpu - oracle| / max|oracle| <= 1e-12 over the interior
after several steps.  Graph replay, per-stage calls and chunking are bitwise
identical to eager full steps.
"""
import numpy as np
import pytest

import sympygr_b200 as sg
from oracle import pyoracle as po
from sympygr_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
SIGMA = 0.2


def _batch(flags, seed=7):
    from test_gpu_parity import _fake_batch

    sizes = [13, 16, 21, 13, 25]
    return _fake_batch(list(zip(sizes, flags)), seed=seed)


def _gpu_evolve(ctx, u, blocks, dt, steps, precision=sg.FP64, chunk_points=0, mode="step"):
    import torch

    plan = sg.Plan(ctx, blocks, precision, chunk_points)
    rk = sg.RK4(plan)
    ud = torch.from_numpy(u).cuda()
    cols = list(ud)
    prm = sg.Params.make(ko_sigma=SIGMA, precision=precision)
    rk.init(cols)
    if mode == "step":
        for _ in range(steps):
            rk.step(cols, dt, prm)
    elif mode == "stage":
        for _ in range(steps):
            for st in range(4):
                rk.stage(st, cols, dt, prm)
    else:  # graph of all steps
        rk.capture(cols, dt, prm, steps)
        assert rk.graph_steps == steps
        rk.launch()
    torch.cuda.synchronize()
    out = ud.cpu().numpy()
    rk.close()
    plan.close()
    return out


@pytest.mark.parametrize("flags", [(0x3F,) * 5, (0, 0x15, 0x3F, 0x2A, 0x08)])
def test_rk4_vs_oracle(ctx, oracle_lib, flags):
    u, blocks, total = _batch(flags)
    dt, steps = 2e-3, 3
    ref = u.copy()
    orc = po.OracleRK4(blocks, total, po.params(ko_sigma=SIGMA))
    orc.init(ref)
    for _ in range(steps):
        orc.step(ref, dt)
    got = _gpu_evolve(ctx, u, blocks, dt, steps)
    m = orc.mask
    assert np.array_equal(got[:, ~m], u[:, ~m])  # only interior points are written
    mx, _ = po.rel_errors(got[:, m], ref[:, m])
    assert mx.max() < TOL64, (mx.max(), int(np.argmax(mx)))
    # and the state moved: the comparison is not trivially of the initial data
    assert np.abs(got[:, m] - u[:, m]).max() > 1e-3


def test_rk4_graph_stage_and_chunking_are_bitwise_identical(ctx):
    u, blocks, total = _batch((0x3F, 0, 0x15, 0x3F, 0x21), seed=9)
    dt, steps = 1e-3, 2
    ref = _gpu_evolve(ctx, u, blocks, dt, steps, mode="step")
    assert np.array_equal(ref, _gpu_evolve(ctx, u, blocks, dt, steps, mode="stage"))
    assert np.array_equal(ref, _gpu_evolve(ctx, u, blocks, dt, steps, mode="graph"))
    assert np.array_equal(ref, _gpu_evolve(ctx, u, blocks, dt, steps, chunk_points=4000))
    assert np.array_equal(ref, _gpu_evolve(ctx, u, blocks, dt, steps, chunk_points=4000,
                                           mode="graph"))


def test_rk4_all_faces_flagged_ignores_ghosts(ctx):
    """With bflag 0x3F every block is self-contained: perturbing the ghost layer of
    the state changes nothing in the evolved interior."""
    u, blocks, total = _batch((0x3F,) * 5, seed=4)
    mask = po.interior_elements(blocks, total)
    inside = np.zeros(total, dtype=bool)
    for b in blocks:
        inside[b.offset:b.offset + b.npad] = True
    ghosts = inside & ~mask
    u2 = u.copy()
    u2[:, ghosts] += np.random.default_rng(0).uniform(-0.5, 0.5, (24, int(ghosts.sum())))
    a = _gpu_evolve(ctx, u, blocks, 2e-3, 3)
    b = _gpu_evolve(ctx, u2, blocks, 2e-3, 3)
    assert np.array_equal(a[:, mask], b[:, mask])


def test_rk4_mixed_tracks_fp64(ctx):
    sizes, counts = (13, 21, 37), (12, 6, 2)
    u, blocks = wl.two_puncture_batch(sizes, counts, seed=5)
    blocks = [wl.Block(b.offset, b.sz, 0x3F, b.pmin, b.pmax) for b in blocks]
    dt = 0.25 * min(b.h[0] for b in blocks)
    a = _gpu_evolve(ctx, u, blocks, dt, 4, sg.FP64)
    b = _gpu_evolve(ctx, u, blocks, dt, 4, sg.MIXED)
    m = po.interior_elements(blocks, u.shape[1])
    # compare the change over the run, the part the RHS precision can affect
    da, db = a[:, m] - u[:, m], b[:, m] - u[:, m]
    for v in range(24):
        s = np.abs(da[v]).max()
        if s > 0:
            assert np.abs(da[v] - db[v]).max() / s < 1e-5, v


def test_rk4_errors_are_reported(ctx):
    import torch

    u, blocks, total = _batch((0x3F,) * 5)
    plan = sg.Plan(ctx, blocks, sg.FP64)
    rk = sg.RK4(plan)
    ud = torch.from_numpy(u).cuda()
    for bad in (lambda: rk.step(list(ud), -1.0, sg.Params.make()),
                lambda: rk.step(list(ud), 1e-3, sg.Params.make(precision=sg.MIXED)),
                lambda: rk.stage(4, list(ud), 1e-3, sg.Params.make()),
                lambda: rk.launch()):
        with pytest.raises(sg.B200BssnError) as ei:
            bad()
        assert ei.value.code == -1
    rk.close()
    plan.close()


def test_evolve_checkpoint_resume_is_bitwise(tmp_path):
    """4 steps straight through equal 2 steps, a checkpoint, and 2 resumed steps."""
    from sympygr_b200 import evolve

    common = ["--scale", "0.01", "--check-every", "2", "--graph-steps", "2", "--precisions", "fp64"]
    a, b, c = (str(tmp_path / k) for k in "abc")
    evolve.main(common + ["--steps", "4", "--checkpoint", a])
    evolve.main(common + ["--steps", "2", "--checkpoint", b])
    out = evolve.main(common + ["--steps", "2", "--resume", b + "/fp64", "--checkpoint", c])
    sa, _, ma = evolve.load_checkpoint(a + "/fp64")
    sc, _, mc = evolve.load_checkpoint(c + "/fp64")
    assert ma["step"] == mc["step"] == 4
    assert np.array_equal(sa, sc)
    assert out["runs"]["fp64"]["finite"]
    assert out["runs"]["fp64"]["history"][-1]["step"] == 4


def test_evolve_tiled_domain_with_sommerfeld_faces(tmp_path):
    """A cube domain tiled by 2^3 blocks, Sommerfeld faces on its outer boundary only:
    both precisions stay finite and mixed follows FP64."""
    from sympygr_b200 import evolve

    out = evolve.main(["--layout", "tiled", "--tiles", "2", "--tile-size", "21", "--half-width", "8",
                       "--steps", "6", "--check-every", "3", "--graph-steps", "3",
                       "--json", str(tmp_path / "t.json")])
    assert out["boundary"] == "domain"
    for name in ("fp64", "mixed"):
        assert out["runs"][name]["finite"] and out["runs"][name]["steps"] == 6
    assert max(c["max_rel"] for c in out["mixed_vs_fp64_change"]) < 1e-4
    assert abs(out["ham_growth_ratio_mixed_over_fp64"] - 1.0) < 1e-3
