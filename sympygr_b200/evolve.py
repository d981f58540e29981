"""RK4 evolution of the two-puncture block batch on one GPU, FP64 against mixed.

The batch is the octree-like two-puncture Brill-Lindquist set of
``workloads.two_puncture_batch`` (3000 blocks, padded sizes 13..135, ~1.07e8
interior points at --scale 1).  Its blocks overlap at random positions, so there is
no ghost exchange: every block evolves on its own, and the ghost points of the
state keep the initial data (Dirichlet data from the exact initial slice).
``--boundary`` picks the faces that get the reference's one-sided closures and
Sommerfeld values (bssn/src/rhs.cpp:833-977):

* ``frozen`` (default): none; centred stencils read the frozen ghost data;
* ``batch``: the batch's own face masks (10 % of the blocks, random faces);
* ``all``: all six faces of every block (bflag 0x3F).

On faces inside the strong-field region the reference's closure + Sommerfeld
treatment grows exponentially (its own right-hand side shows it: K grows ~2.5x every
5 steps next to one flagged face of a 37^3 block, at any KO strength), so the
100-step comparison of the batch runs with ``frozen``; the other two modes show that
growth and that mixed precision follows FP64 through it.

``--layout tiled`` evolves instead a cube domain [-L, L]^3 (``--half-width``) tiled
by ``--tiles``^3 blocks of padded size ``--tile-size`` around the same two punctures:
the faces on the domain boundary carry the Sommerfeld values and one-sided closures
(their bflag bits), the faces between blocks keep the frozen initial ghost data (the
ghost exchange between blocks is outside this path).  dt = CFL * the smallest spacing.  The whole step loop runs as replays of a CUDA graph of
``--graph-steps`` RK4 steps (each step: 4 stages x 3 launches per chunk, the stage
update fused into the algebra kernel).  Every ``--check-every`` steps the driver
evaluates the Hamiltonian and momentum constraints on the device (per-block sums of
squares and maxima) and reads the lapse at the grid points nearest the two
punctures.

Checkpoints (``--checkpoint DIR``) are a raw dump of the final state of each run
(``DIR/<precision>/state.npy``, [24, n] float64) with the block table, step count and
run settings (``meta.json``); ``--resume DIR/<precision>`` continues such a run.

Reported per precision: steps/s of the stepping alone and of the whole loop with
checks, RHS evaluations per second in Mpoints/s, the constraint L2 norms and their
growth over the run, the lapse history at the punctures; and, mixed against FP64,
the per-variable max and RMS relative difference of the final state's change over
the run.

    python -m sympygr_b200.evolve --steps 100 --json evolve.json
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import capi
from . import workloads as wl

PUNCTURES = ((-4.0, 0.0, 0.0), (4.0, 0.0, 0.0))


def scaled_counts(scale: float):
    return tuple(max(1, int(round(c * scale))) for c in wl.BATCH_COUNTS)


def nearest_points(blocks, targets):
    """For each target (x, y, z): the element index of the nearest interior grid point
    over all blocks, and that point's coordinates."""
    out = []
    for t in targets:
        best = (math.inf, -1, None)
        for b in blocks:
            h = b.h
            idx, pos = [], []
            for a in range(3):
                i = int(round((t[a] - b.pmin[a]) / h[a]))
                i = min(max(i, 3), b.sz[a] - 4)
                idx.append(i)
                pos.append(b.pmin[a] + i * h[a])
            d = math.dist(pos, t)
            if d < best[0]:
                e = b.offset + idx[0] + b.sz[0] * (idx[1] + b.sz[1] * idx[2])
                best = (d, e, tuple(pos))
        out.append((best[1], best[2]))
    return out


def constraint_l2(norms: np.ndarray, points: int):
    """Global L2 (RMS over interior points) and max of ham, mom0..2 from the
    per-block [sum of squares x4, max x4] table."""
    nb = norms.reshape(-1, 8)
    l2 = np.sqrt(nb[:, :4].sum(axis=0) / points)
    mx = nb[:, 4:].max(axis=0)
    return l2, mx


def save_checkpoint(path: str, u, blocks, meta: dict):
    """Raw dump of the state ([24, n] float64) plus the block table and run settings."""
    import os

    os.makedirs(path, exist_ok=True)
    arr = u.cpu().numpy() if hasattr(u, "cpu") else np.asarray(u)
    np.save(os.path.join(path, "state.npy"), arr)
    meta = dict(meta)
    meta["blocks"] = [{"offset": b.offset, "sz": list(b.sz), "bflag": b.bflag, "pmin": list(b.pmin),
                       "pmax": list(b.pmax)} for b in blocks]
    with open(os.path.join(path, "meta.json"), "w") as f:
        json.dump(meta, f)


def load_checkpoint(path: str):
    """(state [24, n] float64, block list, settings) of a checkpoint directory."""
    import os

    with open(os.path.join(path, "meta.json")) as f:
        meta = json.load(f)
    blocks = [wl.Block(b["offset"], tuple(b["sz"]), b["bflag"], tuple(b["pmin"]), tuple(b["pmax"]))
              for b in meta.pop("blocks")]
    return np.load(os.path.join(path, "state.npy")), blocks, meta


def run_precision(ctx, u0, blocks, precision, args, probes, dt, step0: int = 0):
    import torch

    plan = capi.Plan(ctx, blocks, precision, args.chunk_points)
    rk = capi.RK4(plan)
    u = u0.clone()
    cols = list(u)
    prm = capi.Params.make(ko_sigma=args.ko_sigma, precision=precision)
    norms = torch.zeros(len(blocks) * 8, dtype=torch.float64, device=u.device)
    rk.init(cols)
    stream = torch.cuda.ExternalStream(ctx.stream)
    probe_idx = torch.tensor([p[0] for p in probes], dtype=torch.int64, device=u.device)

    history = []

    def check(step):
        plan.constraints_device(cols, None, norms)
        with torch.cuda.stream(stream):
            nb = norms.cpu().numpy()  # ordered after the constraint kernels on ctx.stream
            lapse = u[wl.U_ALPHA].index_select(0, probe_idx).cpu().numpy()
        l2, mx = constraint_l2(nb, plan.points)
        history.append({"step": step0 + step, "t": (step0 + step) * dt, "ham_l2": l2[0],
                        "mom_l2": l2[1:].tolist(),
                        "ham_max": mx[0], "mom_max": mx[1:].tolist(), "lapse": lapse.tolist(),
                        "finite": bool(np.isfinite(nb).all())})
        return history[-1]

    g = max(1, min(args.graph_steps, args.check_every, args.steps))
    rk.capture(cols, dt, prm, g)
    check(0)
    # stepping alone: CUDA events on the context stream around each graph replay
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms = 0.0
    done = 0
    wall0 = time.perf_counter()
    while done < args.steps:
        n = min(g, args.steps - done)
        if n != g:  # tail shorter than the graph: capture it once
            rk.capture(cols, dt, prm, n)
        ev0.record(stream)
        rk.launch()
        ev1.record(stream)
        ev1.synchronize()
        step_ms += ev0.elapsed_time(ev1)
        done += n
        if done % args.check_every == 0 or done == args.steps:
            h = check(done)
            if not h["finite"]:
                break
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    bad = plan.check_finite(cols)  # NaN/Inf guard over the final state
    final = u.cpu()  # host copy: frees HBM for the next run
    del u, cols
    rk.close()
    plan.close()
    pts = sum(b.ninterior for b in blocks)
    return {
        "precision": "mixed" if precision == capi.MIXED else "fp64",
        "steps": done,
        "step0": step0,
        "finite": bad is None,
        "dt": dt,
        "graph_steps": g,
        "step_seconds": step_ms / 1e3,
        "steps_per_s": done / (step_ms / 1e3),
        "steps_per_s_with_checks": done / wall,
        "rhs_mpoints_per_s": 4 * done * pts / (step_ms / 1e3) / 1e6,
        "history": history,
        "ham_l2_growth": history[-1]["ham_l2"] / history[0]["ham_l2"],
        "mom_l2_final": history[-1]["mom_l2"],
    }, final


def main(argv=None):
    import torch

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--cfl", type=float, default=0.25)
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the 3000-block batch")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ko-sigma", type=float, default=0.4)
    ap.add_argument("--check-every", type=int, default=10)
    ap.add_argument("--graph-steps", type=int, default=10)
    ap.add_argument("--chunk-points", type=int, default=0)
    ap.add_argument("--precisions", default="fp64,mixed")
    ap.add_argument("--boundary", default="frozen", choices=["frozen", "batch", "all"],
                    help="face flags of the batch layout")
    ap.add_argument("--layout", default="batch", choices=["batch", "tiled"])
    ap.add_argument("--tiles", type=int, default=4, help="tiled layout: blocks per axis")
    ap.add_argument("--tile-size", type=int, default=37, help="tiled layout: padded block size")
    ap.add_argument("--half-width", type=float, default=8.0, help="tiled layout: domain [-L, L]^3")
    ap.add_argument("--checkpoint", default="", help="directory for the final states")
    ap.add_argument("--resume", default="", help="checkpoint directory of one precision to continue")
    ap.add_argument("--json", default="")
    args = ap.parse_args(argv)

    ctx = capi.Context(0)
    step0 = 0
    if args.resume:
        state, blocks, meta = load_checkpoint(args.resume)
        u0 = torch.from_numpy(state).cuda()
        step0 = int(meta["step"])
        dt = float(meta["dt"])
        args.precisions = meta["precision"]
        args.boundary = meta["boundary"]
    elif args.layout == "tiled":
        blocks, total = wl.tiled_domain_blocks(args.tiles, args.tile_size, args.half_width)
        u0 = wl.two_puncture_fields_torch(blocks, total, device="cuda")
        args.boundary = "domain"
        dt = args.cfl * min(min(b.h) for b in blocks)
    else:
        u0, blocks = wl.two_puncture_batch_torch(wl.BATCH_SIZES, scaled_counts(args.scale), args.seed,
                                                 device="cuda")
        if args.boundary != "batch":
            flag = 0x3F if args.boundary == "all" else 0
            blocks = [wl.Block(b.offset, b.sz, flag, b.pmin, b.pmax) for b in blocks]
        dt = args.cfl * min(min(b.h) for b in blocks)
    torch.cuda.empty_cache()  # drop the initial-data temporaries before the big buffers
    probes = nearest_points(blocks, PUNCTURES)
    mask = torch.zeros(u0.shape[1], dtype=torch.bool, device="cuda")
    for b in blocks:
        nx, ny, nz = b.sz
        seg = mask[b.offset:b.offset + b.npad].view(nz, ny, nx)
        seg[3:-3, 3:-3, 3:-3] = True
    if args.layout == "tiled" and not args.resume:
        workload = (f"two-puncture tiled domain [-{args.half_width:g}, {args.half_width:g}]^3, "
                    f"{args.tiles}^3 blocks of {args.tile_size}^3")
    else:
        workload = f"two-puncture batch x{args.scale:g}, {len(blocks)} blocks"
    out = {"workload": workload,
           "boundary": args.boundary,
           "points": sum(b.ninterior for b in blocks), "dt": dt, "cfl": args.cfl,
           "probes": [{"target": t, "point": p[1]} for t, p in zip(PUNCTURES, probes)],
           "runs": {}}
    finals = {}
    for name in args.precisions.split(","):
        prec = capi.MIXED if name == "mixed" else capi.FP64
        res, fin = run_precision(ctx, u0, blocks, prec, args, probes, dt, step0)
        out["runs"][name] = res
        finals[name] = fin
        if args.checkpoint:
            import os

            save_checkpoint(os.path.join(args.checkpoint, name), fin, blocks,
                            {"precision": name, "step": step0 + res["steps"], "dt": dt,
                             "boundary": args.boundary, "ko_sigma": args.ko_sigma,
                             "scale": args.scale, "seed": args.seed})
        print(json.dumps({k: v for k, v in res.items() if k != "history"}), flush=True)
    if "fp64" in finals and "mixed" in finals:
        a, b = finals["fp64"], finals["mixed"]
        cmp = []
        for v in range(24):
            da = (a[v].cuda() - u0[v])[mask]
            db = (b[v].cuda() - u0[v])[mask]
            s = da.abs().max().item()
            diff = (da - db).abs()
            cmp.append({"var": wl.VAR_NAMES[v],
                        "max_rel": diff.max().item() / s if s > 0 else 0.0,
                        "rms_rel": diff.pow(2).mean().sqrt().item() / s if s > 0 else 0.0})
        out["mixed_vs_fp64_change"] = cmp
        hf, hm = out["runs"]["fp64"], out["runs"]["mixed"]
        out["ham_growth_ratio_mixed_over_fp64"] = hm["ham_l2_growth"] / hf["ham_l2_growth"]
        out["lapse_final"] = {"fp64": hf["history"][-1]["lapse"], "mixed": hm["history"][-1]["lapse"]}
    if args.json:
        with open(args.json, "w") as f:
            json.dump(out, f, indent=1)
    summary = {k: v for k, v in out.items() if k not in ("runs", "mixed_vs_fp64_change")}
    if "mixed_vs_fp64_change" in out:
        summary["max_rel_change_diff"] = max(c["max_rel"] for c in out["mixed_vs_fp64_change"])
    print(json.dumps(summary), flush=True)
    ctx.close()
    return out


if __name__ == "__main__":
    main()
