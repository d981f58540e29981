"""Small profiling case for ncu: four 69^3 blocks and one 135^3 block of the
two-puncture batch (3.15M interior points, ~0.6 GB per 24-variable state, larger
than L2), evaluated twice with one plan.

    python -m sympygr_b200.profile_case [mixed|fp64]
"""
import sys

import torch

import sympygr_b200 as sg
from sympygr_b200 import workloads as wl


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    prec = sg.FP64 if (argv and argv[0] == "fp64") else sg.MIXED
    u, blocks = wl.two_puncture_batch_torch((69, 135), (4, 1), seed=0, device="cuda")
    rhs = torch.zeros_like(u)
    ctx = sg.Context(0)
    plan = sg.Plan(ctx, blocks, prec)
    prm = sg.Params.make(ko_sigma=0.4, precision=prec)
    for _ in range(2):
        plan.rhs_device(list(rhs), list(u), prm)
    torch.cuda.synchronize()
    print("points", plan.points, "launches", plan.launches, "ok")
    plan.close()
    ctx.close()


if __name__ == "__main__":
    main()
