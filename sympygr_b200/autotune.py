"""Autotuner: per block-size class, the plan knobs that evaluate the right-hand side
fastest on this GPU.

For each padded size class of the two-puncture batch (13, 21, 37, 69, 135; the
class's block count from the batch, times --scale) it builds a plan of that class
alone and times one evaluation (CUDA events, device-resident inputs larger than L2)
for every candidate of

* tile shape: 16 x tile_y columns per derivative CTA, tile_y 4, 8 or 16 (64, 128 or
  256 threads; the staged plane, the D_x halo rows and the register queues follow);
* registers-per-thread split of the derivative kernels: 96 / 128 registers for the kinds
  without / with second derivatives, one CTA per SM more (80 / 96) or one fewer
  (128 / 168) -- with 16x8 tiles (the plans' default is the last for FP64, the first
  for MIXED);
* output points per thread: one, or two (y pairs of 16x16 tiles in CTAs of 128 threads);
* slab depth (staging depth along z): the z-planes per work unit of the derivative
  kernel (candidates that cut the interior into the same number of slabs are the same
  plan, so one per slab count is timed);
* with --ctas, derivative CTAs per SM capped at 1 or 2 as well as uncapped.

It writes the per-class table and choice to JSON.  ``tuned_plan`` builds a plan for
any block list from such a table: each block gets its class's slab depth
(b200bssn_plan_options.block_slab_depth); the tile shape, register split and CTA
count are plan-wide knobs.  They are settled on the whole batch: the default plan, the
per-class depths with the default plan-wide knobs, and the per-class depths with the
knobs of the class holding the most points are timed, and the table keeps the fastest
(so a class's win inside the timing noise cannot cost the other classes).

    python -m sympygr_b200.autotune --precision mixed --json tune_mixed.json
"""
from __future__ import annotations

import argparse
import json

from . import capi
from . import workloads as wl


def depth_candidates(n: int):
    """One depth per distinct slab count of an n^3 block (interior n-6 planes)."""
    planes = n - 6
    out, seen = [], set()
    for d in (8, 12, 16, 24, 32, 40, 48, 64, 96, 128, planes):
        d = min(d, planes)
        ns = -(-planes // d)
        if ns not in seen:
            seen.add(ns)
            out.append(d)
    return out


def time_plan(plan, rhs, u, prm, reps: int = 5, warmup: int = 2) -> float:
    """Milliseconds per evaluation (CUDA events on the context stream)."""
    import torch

    stream = torch.cuda.ExternalStream(plan.ctx.stream)
    for _ in range(warmup):
        plan.rhs_device(rhs, u, prm)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        plan.rhs_device(rhs, u, prm)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


# (tile_y, deriv_regs) variants of the derivative kernels built into the library
# (deriv_regs 1: 96/128 registers for the kinds without/with second derivatives, 2: 80/96,
# 3: 128/168)
KERNEL_VARIANTS = [(8, 1, 1), (4, 1, 1), (16, 1, 1), (8, 2, 1), (8, 3, 1), (16, 0, 2)]  # + points per thread


def tuned_plan(ctx, blocks, precision, table, chunk_points: int = 0):
    """A plan whose blocks use their size class's tuned slab depth and the table's
    plan-wide knobs (the default plan where the table found the tuned one no faster)."""
    if table.get("use_default_plan"):
        return capi.Plan(ctx, blocks, precision, chunk_points)
    choice = {int(k): v for k, v in table["choice"].items()}
    depths = [choice.get(b.sz[2], {}).get("slab_depth", 0) for b in blocks]
    return capi.Plan(ctx, blocks, precision, chunk_points, deriv_ctas_per_sm=table["deriv_ctas_per_sm"],
                     block_slab_depth=depths, tile_y=table.get("tile_y", 0),
                     deriv_regs=table.get("deriv_regs", 0), points_per_thread=table.get("points_per_thread", 0))


def main(argv=None):
    import torch

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--json", default="")
    ap.add_argument("--ctas", action="store_true", help="also sweep CTA caps of 1 and 2 per SM")
    args = ap.parse_args(argv)
    prec = capi.MIXED if args.precision == "mixed" else capi.FP64
    prm = capi.Params.make(ko_sigma=0.4, precision=prec)
    ctx = capi.Context(0)
    counts = tuple(max(1, int(round(c * args.scale))) for c in wl.BATCH_COUNTS)
    table = {"precision": args.precision, "classes": {}, "choice": {}}
    best_points = (0, None)
    for n, c in zip(wl.BATCH_SIZES, counts):
        u, blocks = wl.two_puncture_batch_torch((n,), (c,), seed=1, device="cuda")
        rhs = torch.zeros_like(u)
        pts = sum(b.ninterior for b in blocks)
        rows = []
        for ty, regs, ppt in KERNEL_VARIANTS:
            for d in depth_candidates(n):
                for ctas in ((0, 1, 2) if args.ctas else (0,)):
                    plan = capi.Plan(ctx, blocks, prec, slab_depth=d, deriv_ctas_per_sm=ctas, tile_y=ty,
                                     deriv_regs=regs, points_per_thread=ppt)
                    ms = time_plan(plan, list(rhs), list(u), prm, args.reps)
                    plan.close()
                    rows.append({"tile_y": ty, "deriv_regs": regs, "points_per_thread": ppt, "slab_depth": d,
                                 "deriv_ctas_per_sm": ctas, "ms": ms, "mpts_per_s": pts / ms / 1e3})
                    print(json.dumps({"class": n, **rows[-1]}), flush=True)
        best = max(rows, key=lambda r: r["mpts_per_s"])
        nslab = lambda d: -(-(n - 6) // d)  # noqa: E731 -- slabs of the class's blocks at depth d
        dregs = 3 if prec == capi.FP64 else 1  # the plan's default split for this precision
        default = next(r for r in rows if r["tile_y"] == 8 and r["deriv_regs"] == dregs and r["deriv_ctas_per_sm"] == 0
                       and r["points_per_thread"] == 1 and nslab(r["slab_depth"]) == nslab(48))
        table["classes"][str(n)] = {"blocks": c, "points": pts, "runs": rows}
        table["choice"][str(n)] = {k: best[k] for k in ("tile_y", "deriv_regs", "points_per_thread", "slab_depth",
                                                        "deriv_ctas_per_sm", "mpts_per_s")}
        table["choice"][str(n)]["gain_over_default"] = best["mpts_per_s"] / default["mpts_per_s"]
        if pts > best_points[0]:
            best_points = (pts, best)
        del u, rhs
        torch.cuda.empty_cache()
    # the whole batch settles the plan-wide knobs: the default plan, the per-class depths
    # with the default knobs, and the per-class depths with the knobs of the class
    # holding the most points
    knobs = ("deriv_ctas_per_sm", "tile_y", "deriv_regs", "points_per_thread")
    u, blocks = wl.two_puncture_batch_torch(wl.BATCH_SIZES, counts, seed=0, device="cuda")
    rhs = torch.zeros_like(u)
    pts = sum(b.ninterior for b in blocks)
    plan = capi.Plan(ctx, blocks, prec)
    ms_default = time_plan(plan, list(rhs), list(u), prm, args.reps)
    plan.close()
    candidates = {"default_knobs": {k: 0 for k in knobs},
                  "class_knobs": {k: best_points[1][k] for k in knobs}}
    timed = {}
    for name, kn in candidates.items():
        table.update(kn)
        plan = tuned_plan(ctx, blocks, prec, table)
        timed[name] = time_plan(plan, list(rhs), list(u), prm, args.reps)
        plan.close()
    pick = min(timed, key=timed.get)
    table.update(candidates[pick])
    table["use_default_plan"] = ms_default <= timed[pick]  # the tuned depths did not pay
    table["batch"] = {"points": pts, "default_mpts_per_s": pts / ms_default / 1e3,
                      "depths_default_knobs_mpts_per_s": pts / timed["default_knobs"] / 1e3,
                      "depths_class_knobs_mpts_per_s": pts / timed["class_knobs"] / 1e3,
                      "tuned_mpts_per_s": pts / min(ms_default, timed[pick]) / 1e3, "plan_wide": pick}
    print(json.dumps({"choice": table["choice"], "batch": table["batch"],
                      "plan_wide": {k: table[k] for k in ("deriv_ctas_per_sm", "tile_y", "deriv_regs",
                                                          "points_per_thread")}}),
          flush=True)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(table, f, indent=1)
    ctx.close()
    return table


if __name__ == "__main__":
    main()
