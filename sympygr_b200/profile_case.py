"""Small profiling case for ncu: four 69^3 blocks and one 135^3 block of the
two-puncture batch, one of them with a flagged face (3.15M interior points,
~0.6 GB per 24-variable state, larger than L2), evaluated twice with one plan;
with ``--steps`` also the constraint kernel once and that many RK4 steps (4
stages each: the algebra kernel in its three RK4 stage modes).

    python -m sympygr_b200.profile_case [mixed|fp64] [--steps N]
"""
import argparse

import torch

import sympygr_b200 as sg
from sympygr_b200 import workloads as wl


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("precision", nargs="?", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--steps", type=int, default=0)
    args = ap.parse_args(argv)
    prec = sg.FP64 if args.precision == "fp64" else sg.MIXED
    # seed 5: one of the 69^3 blocks has a flagged face (8 % of the points), like the
    # 3000-block batch (about 10 % of its points lie in blocks with flagged faces)
    u, blocks = wl.two_puncture_batch_torch((69, 135), (4, 1), seed=5, device="cuda")
    rhs = torch.zeros_like(u)
    ctx = sg.Context(0)
    plan = sg.Plan(ctx, blocks, prec)
    prm = sg.Params.make(ko_sigma=0.4, precision=prec)
    for _ in range(2):
        plan.rhs_device(list(rhs), list(u), prm)
    if args.steps:
        norms = torch.zeros(len(blocks) * 8, dtype=torch.float64, device="cuda")
        plan.constraints_device(list(u), None, norms)
        rk = sg.RK4(plan)
        rk.init(list(u))
        for _ in range(args.steps):
            rk.step(list(u), 1e-3, prm)
        torch.cuda.synchronize()
        rk.close()
    torch.cuda.synchronize()
    print("points", plan.points, "launches", plan.launches, "ok")
    plan.close()
    ctx.close()


if __name__ == "__main__":
    main()
