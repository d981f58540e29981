#!/usr/bin/env python
"""Benchmark: batched BSSN right-hand side on B200, mixed precision vs plain FP64.

Workload (one "step" = one RHS evaluation of the whole batch): the octree-like
two-puncture Brill-Lindquist batch of 3000 blocks, padded sizes 13/21/37/69/135
(1800/750/300/120/30 blocks), 1.065e8 interior points, KO sigma 0.4, inputs
resident in HBM (26.7 GB per 24-variable state, far larger than the 126 MB L2, so
no flush is needed between steps).  `value` is the MIXED-precision throughput
(FP64 state and stencils, FP32 algebra) in interior Mpoints/s; the plain FP64
path is timed the same way and reported beside it.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU (torchrun): every rank evaluates its own batch (weak scaling, no
collective on the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "BSSN RHS Mpoints/s, mixed vs plain FP64 on 1 B200 at <=1e-6 rel err; %roofline"
UNIT = "Mpoints/s"
SIGMA = 0.4
# the workload both arms report (the precision of each is in its `dtype`)
WORKLOAD = ("two-puncture Brill-Lindquist batch: 3000 blocks, padded 13/21/37/69/135 "
            "(1800/750/300/120/30), KO sigma 0.4")
# Algorithmic work per interior point.  Algebra: the operation count of the staged,
# generated device function (sympy count_ops, an FMA counted as 2) plus the KO add
# (2 per variable) and the eta damping (~10).  Derivatives: 72 first derivatives
# x 12 flops (6-point stencil, multiply-add each), 33 second derivatives x 14,
# 33 mixed (a first derivative of a first derivative) x 12, KO 72 x 14.
ALGEBRA_FLOPS_PER_POINT = 2428 + 48 + 10
DERIV_FLOPS_PER_POINT = 72 * 12 + 33 * 14 + 33 * 12 + 72 * 14
MIXED_BAR = 1e-6
# Algorithmic bytes per interior point.  Derivative kernel: reads the 24 state
# variables over the padded blocks (24 x 8 B x padded/interior points of the
# batch) and writes the scratch (138 derivative slots and 24 KO sums, x 8 B in FP64
# or x 4 B in MIXED).  Algebra kernel: reads the state at the point (24 x 8 B) and the scratch,
# writes 24 x 8 B.
SCRATCH_BYTES = {"fp64": 138 * 8 + 24 * 8, "mixed": 138 * 4 + 24 * 4}
# DRAM bytes per interior point of each kernel measured by ncu on a large-block case
# (profiles/ncu_derivs_algebra_large_blocks.md): derivative stage (its two kernels,
# variables without + with second derivatives) / algebra kernel.
NCU_TRAFFIC_PER_POINT = {"mixed": (376.0 + 646.0, 1123.0), "fp64": (584.0 + 1122.0, 2110.0)}

PG_TIMEOUT_S = 120  # process-group timeout under torchrun (N > 1)


def max_over_ranks(value: float, dist=None, device="cuda") -> float:
    """The largest `value` over all ranks (every rank receives it); `dist` None: one process."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def sum_over_ranks(value: int, dist=None, device="cuda") -> int:
    """The sum of an integer count over all ranks; `dist` None: one process."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def duplex_copy_gbs(h_src, h_dst, n: int = 128 * 1024 * 1024, reps: int = 3) -> float:
    """GB/s per direction of a host->device and a device->host copy running at once
    (pinned host memory, one stream per direction, `n` elements each): the transfer
    bound of the host-buffer path, which moves its state in and its RHS out concurrently."""
    import torch

    n = min(n, h_src.numel(), h_dst.numel())
    src, dst = h_src.view(-1)[:n], h_dst.view(-1)[:n]
    d_in = torch.empty(n, dtype=src.dtype, device="cuda")
    d_out = torch.zeros(n, dtype=src.dtype, device="cuda")
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    cur = torch.cuda.current_stream()

    def once(k):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        s_in.wait_event(e0)
        s_out.wait_event(e0)
        for _ in range(k):
            with torch.cuda.stream(s_in):
                d_in.copy_(src, non_blocking=True)
            with torch.cuda.stream(s_out):
                dst.copy_(d_out, non_blocking=True)
        cur.wait_stream(s_in)
        cur.wait_stream(s_out)
        e1.record(cur)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3

    once(1)
    secs = once(reps)
    del d_in, d_out
    return reps * n * src.element_size() / secs / 1e9


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons, power = [], None, set(), []
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                  "sw_power_cap"], f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def stratified_blocks(blocks, frac):
    """A class-proportional subset of a block list (at least one block per class)."""
    by = {}
    for b in blocks:
        by.setdefault(b.sz[0], []).append(b)
    out = []
    for n, bl in sorted(by.items()):
        m = max(1, int(round(len(bl) * frac)))
        out.extend(bl[:m])
    return out


def cpu_reference_run(u_host, blocks, nthreads):
    """The reference's own CPU bssnrhs (compiled from its sources, -O3) over a block
    list in its block-parallel OpenMP loop; returns (seconds, interior points)."""
    import numpy as np

    from oracle import pyoracle as po

    rhs = np.zeros_like(u_host)
    prm = po.params(ko_sigma=SIGMA)
    secs = po.ref_blocks_omp(u_host, rhs, blocks, prm, nthreads=nthreads, flavour="fast")
    return secs, sum(b.ninterior for b in blocks)


def compact_host_batch(blocks):
    """Host arrays for a block subset, re-offset compactly (numpy generator)."""
    import numpy as np

    from sympygr_b200 import workloads as wl

    out, off = [], 0
    for b in blocks:
        out.append(wl.Block(off, b.sz, b.bflag, b.pmin, b.pmax))
        off += b.npad
    u = np.zeros((24, off))
    punct = [(-4.0, 0.0, 0.0, 0.5), (4.0, 0.0, 0.0, 0.5)]
    for b in out:
        x, y, z = wl.coords(b)
        wl._bl_fields(u, slice(b.offset, b.offset + b.npad), x, y, z, punct)
    return u, out


def host_bytes_available() -> int:
    """MemAvailable of this host (bytes), or the physical memory when /proc is absent."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")


def ref_fraction(args):
    if args.ref_fraction > 0:
        return min(1.0, args.ref_fraction)
    return max(0.1, min(1.0, (os.cpu_count() or 1) / 30.0))


def reference_arm(args, rank, world):
    """`--impl reference`: the reference's CPU bssnrhs on this host's cores."""
    if rank != 0:
        return None
    from oracle import pyoracle as po
    from sympygr_b200 import workloads as wl

    if not po.have_reference("fast"):
        return {"impl": "reference", "unavailable": "reference build oracle/_ref/libbssn_ref_fast.so missing"}
    ncores = os.cpu_count() or 1
    blocks, _ = wl.batch_blocks(seed=0)
    frac = ref_fraction(args)
    sample = stratified_blocks(blocks, frac)
    u, sblocks = compact_host_batch(sample)
    # big blocks first so the block-parallel loop does not end on a long tail
    order = sorted(range(len(sblocks)), key=lambda i: -sblocks[i].npad)
    sblocks = [sblocks[i] for i in order]
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_reference_run(u, sblocks, ncores)
    times, pts = [], 0
    for _ in range(max(1, min(args.steps, 3))):
        s, pts = cpu_reference_run(u, sblocks, ncores)
        times.append(s)
    t = statistics.median(times)
    val = pts / t / 1e6
    sample_desc = (f"{len(sblocks)} of 3000 blocks ({frac:.3g} class-proportional sample, "
                   f"{pts} interior points, largest blocks first) per step; median of {len(times)} steps")
    return {
        "metric": METRIC, "value": round(val, 4), "unit": UNIT, "impl": "reference",
        "n_gpus": world, "steps": len(times), "warmup": min(args.warmup, 1),
        "ms_per_step": round(t * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "blocks": len(blocks),
                   "interior_points_per_gpu": sum(b.ninterior for b in blocks), "sample": sample_desc},
        "cpu_baseline": {"value": round(val, 4), "unit": UNIT, "cores": ncores, "kind": "reference",
                         "sample": sample_desc},
        "e2e": {"value": round(val, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0,
                    help="fraction of the 3000-block batch (1.0 = the benchmark workload)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-upwind", action="store_true", help="skip timing the opt-in upwind mode")
    ap.add_argument("--ref-fraction", type=float, default=0.0,
                    help="class-proportional block sample for the CPU reference; 0 = enough "
                         "135^3 blocks to give every host core one (min 0.1)")
    ap.add_argument("--chunk-points", type=int, default=0)
    ap.add_argument("--slab-depth", type=int, default=0)
    ap.add_argument("--deriv-ctas", type=int, default=0, help="derivative CTAs per SM (0: max)")
    args = ap.parse_args()

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        out = reference_arm(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return

    import numpy as np
    import torch

    import sympygr_b200 as sg
    from sympygr_b200 import capi
    from sympygr_b200 import workloads as wl

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        # short: a rank that died leaves the others with an error at their next
        # collective, not a wait; the longest gap between collectives (pinned staging
        # allocation before the end-to-end timing) is well under it
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=PG_TIMEOUT_S))

    counts = tuple(max(1, int(round(c * args.scale))) for c in wl.BATCH_COUNTS)
    u, blocks = wl.two_puncture_batch_torch(wl.BATCH_SIZES, counts, seed=rank, device="cuda")
    rhs = torch.zeros_like(u)
    ctx = sg.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream)
    plans = {p: sg.Plan(ctx, blocks, p, args.chunk_points, args.slab_depth, args.deriv_ctas)
             for p in (sg.FP64, sg.MIXED)}
    params = {p: sg.Params.make(ko_sigma=SIGMA, precision=p) for p in (sg.FP64, sg.MIXED)}
    npts = plans[sg.FP64].points
    U, R = list(u), list(rhs)

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(prec, k):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            plans[prec].rhs_device(R, U, params[prec])
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1), dist) / k

    for prec in (sg.MIXED, sg.FP64):
        for _ in range(args.warmup):
            plans[prec].rhs_device(R, U, params[prec])
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    clocks.start()
    ms_mixed = timed(sg.MIXED, args.steps)
    clock_info = clocks.stop()
    ms_fp64 = timed(sg.FP64, args.steps)

    # accuracy of the headline path: mixed vs FP64 on the same inputs
    plans[sg.FP64].rhs_device(R, U, params[sg.FP64])
    torch.cuda.synchronize()
    ref64 = rhs.clone()
    plans[sg.MIXED].rhs_device(R, U, params[sg.MIXED])
    torch.cuda.synchronize()
    per_var_max, per_var_rms = [], []
    for v in range(24):  # one variable at a time: no full-size temporaries
        scale = ref64[v].abs().max().item()
        d = rhs[v] - ref64[v]
        rms_ref = ref64[v].square().mean().sqrt().item()
        per_var_max.append(d.abs().max().item() / scale if scale > 0 else 0.0)
        per_var_rms.append(d.square().mean().sqrt().item() / rms_ref if rms_ref > 0 else 0.0)
        del d
    mixed_max_rel = max(per_var_max)
    del ref64

    # per-kernel device time of one evaluation (events between launches)
    prof = {}
    for prec in (sg.MIXED, sg.FP64):
        d_ms, a_ms = plans[prec].profile(R, U, params[prec])
        prof[prec] = (d_ms, a_ms)
    peak64 = capi.fma_peak_tflops(local_rank, sg.FP64)
    peak32 = capi.fma_peak_tflops(local_rank, sg.MIXED)

    # the opt-in upwind mode (4th-order upwind advective derivatives, 72 more scratch
    # slots) on the same batch: one plan at a time, same timing as the headline
    upwind = None
    if not args.no_upwind:
        upwind = {}
        for prec, name in ((sg.MIXED, "mixed"), (sg.FP64, "fp64")):
            p_up = sg.Plan(ctx, blocks, prec, args.chunk_points, args.slab_depth, args.deriv_ctas,
                           advective=True)
            for _ in range(args.warmup):
                p_up.rhs_device(R, U, params[prec])
            barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                p_up.rhs_device(R, U, params[prec])
            e1.record(stream)
            e1.synchronize()
            ms_up = max_over_ranks(e0.elapsed_time(e1), dist) / args.steps
            d_up, a_up = p_up.profile(R, U, params[prec])
            p_up.close()
            upwind[name] = {"value": round(sum_over_ranks(npts, dist) / (ms_up * 1e-3) / 1e6, 3),
                            "ms_per_step": round(ms_up, 3), "deriv_ms": round(d_up, 3),
                            "algebra_ms": round(a_up, 3)}
        torch.cuda.synchronize()

    launches = plans[sg.MIXED].launches * args.steps
    total_pts = sum_over_ranks(npts, dist)  # each rank evaluates its own batch
    val_mixed = total_pts / (ms_mixed * 1e-3) / 1e6
    val_fp64 = total_pts / (ms_fp64 * 1e-3) / 1e6

    d_ms, a_ms = prof[sg.MIXED]
    alg_tf = ALGEBRA_FLOPS_PER_POINT * npts / (a_ms * 1e-3) / 1e12
    d64, a64 = prof[sg.FP64]
    alg64_tf = ALGEBRA_FLOPS_PER_POINT * npts / (a64 * 1e-3) / 1e12
    padded = sum(b.npad for b in blocks)
    read_state = 24 * 8 * padded / npts
    hbm_peak = None
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            hbm_peak = float(json.load(fh)["hbm_gbs"])
        peak_src = "measured (MEASURED_PEAKS.json hbm_gbs, copy test)"
    except Exception:
        hbm_peak, peak_src = 6650.0, "fallback 6.65 TB/s"
    nchunks = max(1, plans[sg.MIXED].launches // 3)  # 3 launches per chunk

    def hbm_roofline(kernel, ms, bytes_per_pt, mode, which):
        gbs = bytes_per_pt * npts / (ms * 1e-3) / 1e9
        traffic = NCU_TRAFFIC_PER_POINT[mode][which] * npts / nchunks
        return {"kernel": kernel, "bound": "hbm", "achieved": round(gbs, 1), "peak": hbm_peak,
                "unit": "GB/s", "frac": round(gbs / hbm_peak, 4), "traffic": round(traffic),
                "bytes_per_point": round(bytes_per_pt, 1), "launches_per_step": nchunks,
                "peak_source": peak_src,
                "traffic_note": ("ncu DRAM bytes/point on a 3.15M-point case x points per chunk "
                                 "(the derivative stage of a chunk is two launches, summed)")}

    # end to end through the host API: H2D of the state, evaluate, D2H of the RHS.  Each
    # rank pins a state and an RHS copy of its batch on the host; where the ranks on this
    # node would need more than 60 % of its available memory, each times a
    # class-proportional sample of its blocks instead (the metric is per point).
    e2e = None
    if not args.no_e2e:
        local = max(1, _env_int("LOCAL_WORLD_SIZE", world))
        span = max(b.offset + b.npad for b in blocks)
        need = 2 * 24 * span * 8
        budget = int(0.6 * host_bytes_available() / local)
        hblocks, hplan, sample_note = blocks, plans[sg.MIXED], None
        if need > budget:
            sub = stratified_blocks(blocks, 0.9 * budget / need)
            hblocks, off = [], 0
            for b in sub:
                hblocks.append(wl.Block(off, b.sz, b.bflag, b.pmin, b.pmax))
                off += b.npad
            u_h = torch.empty((24, off), dtype=u.dtype, pin_memory=True)
            for b, hb in zip(sub, hblocks):
                u_h[:, hb.offset:hb.offset + hb.npad].copy_(u[:, b.offset:b.offset + b.npad])
            span = off
            sample_note = (f"{len(hblocks)} of {len(blocks)} blocks per rank (class-proportional): "
                           f"the full batch's host buffers ({need / 1e9:.1f} GB per rank) exceed "
                           f"60 % of this node's available memory over {local} ranks")
        else:
            u_h = torch.empty(tuple(u.shape), dtype=u.dtype, pin_memory=True)
            u_h.copy_(u)
        del rhs, u
        U = R = None
        torch.cuda.empty_cache()
        if sample_note:
            hplan = sg.Plan(ctx, hblocks, sg.MIXED, args.chunk_points, args.slab_depth, args.deriv_ctas)
        e2e_pts = sum_over_ranks(sum(b.ninterior for b in hblocks), dist)
        r_h = torch.empty(tuple(u_h.shape), dtype=u_h.dtype, pin_memory=True)
        p_host = sg.Params.make(ko_sigma=SIGMA, precision=sg.MIXED, ghost_policy=sg.GHOSTS_ZERO)
        UH, RH = [t.data_ptr() for t in u_h], [t.data_ptr() for t in r_h]
        hplan.rhs_host(RH, UH, span, p_host)  # warm-up (allocates staging)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            hplan.rhs_host(RH, UH, span, p_host)
        e1.record(stream)
        e1.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.e2e_steps, dist)
        nbytes = 24 * span * 8
        # the transfer bound: both directions' bytes at the concurrent copy rate
        gbs = duplex_copy_gbs(u_h, r_h)
        copy_ms = max_over_ranks(nbytes / (gbs * 1e9) * 1e3, dist)
        if sample_note:
            hplan.close()
        del u_h, r_h
        e2e = {"value": round(e2e_pts / (ms * 1e-3) / 1e6, 3), "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "ms_per_step": round(ms, 2), "steps": args.e2e_steps,
               "api": "b200bssn_rhs_plan_host (pinned host arrays, ghosts zeroed)",
               "sample": sample_note,
               "copy_bound": {"duplex_gbs_per_direction": round(gbs, 1),
                              "ms_per_step": round(copy_ms, 2),
                              "value": round(e2e_pts / (copy_ms * 1e-3) / 1e6, 3),
                              "frac": round(copy_ms / ms, 4),
                              "how": "1 GiB H2D and D2H copies at once from/to the same pinned "
                                     "arrays, one stream each; bytes per step / that rate"}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            from oracle import pyoracle as po

            if po.have_reference("fast"):
                frac = ref_fraction(args)
                sample = stratified_blocks(blocks, frac)
                uh, sb = compact_host_batch(sample)
                sb = [sb[i] for i in sorted(range(len(sb)), key=lambda i: -sb[i].npad)]
                secs, pts = cpu_reference_run(uh, sb, os.cpu_count() or 1)
                del uh
                cpu = {"value": round(pts / secs / 1e6, 4), "unit": UNIT, "cores": os.cpu_count(),
                       "kind": "reference",
                       "sample": f"{len(sb)} blocks ({frac:.3g} class-proportional sample of the batch, "
                                 f"{pts} interior points, largest first), one pass, {secs:.2f} s"}
        except Exception as ex:  # the baseline is informational; never fail the bench on it
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {ex}"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": round(val_mixed, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_mixed, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 state+stencils / f32 algebra", "data": "synthetic",
            "config": {"workload": WORKLOAD, "blocks": len(blocks), "interior_points_per_gpu": npts,
                       "l2": "inputs (26.7 GB per state) larger than L2; no flush",
                       "scale": args.scale},
            "fp64": {"value": round(val_fp64, 3), "ms_per_step": round(ms_fp64, 3),
                     "deriv_ms": round(d64, 3), "algebra_ms": round(a64, 3)},
            "mixed_vs_fp64": {"speedup": round(val_mixed / val_fp64, 3),
                              "max_rel_err": mixed_max_rel, "bar": MIXED_BAR,
                              "per_var_max_rel": [float(f"{x:.3g}") for x in per_var_max],
                              "per_var_rms_rel": [float(f"{x:.3g}") for x in per_var_rms]},
            "kernels_ms": {"deriv": round(d_ms, 3), "algebra": round(a_ms, 3)},
            # dominant kernel of the headline (mixed) evaluation: the derivative kernel
            "roofline": hbm_roofline("bssn_derivs_kind_kernel<float,*> (both kinds)", d_ms,
                                     read_state + SCRATCH_BYTES["mixed"], "mixed", 0),
            "roofline_algebra": dict(
                hbm_roofline("bssn_algebra_staged_kernel<float,0>", a_ms,
                             24 * 8 + SCRATCH_BYTES["mixed"] + 24 * 8, "mixed", 1),
                fp32_tflops=round(alg_tf, 3), fp32_peak=round(peak32, 2),
                fp32_frac=round(alg_tf / peak32, 4), flops_per_point=ALGEBRA_FLOPS_PER_POINT,
                fp_peak_source="measured FMA-chain microbenchmark (b200bssn_fma_peak)"),
            "roofline_fp64": {
                "derivs": hbm_roofline("bssn_derivs_kind_kernel<double,*> (both kinds)", d64,
                                       read_state + SCRATCH_BYTES["fp64"], "fp64", 0),
                "algebra": dict(hbm_roofline("bssn_algebra_staged_kernel<double,0>", a64,
                                             24 * 8 + SCRATCH_BYTES["fp64"] + 24 * 8, "fp64", 1),
                                fp64_tflops=round(alg64_tf, 3), fp64_peak=round(peak64, 2),
                                fp64_frac=round(alg64_tf / peak64, 4))},
            "upwind_mode": upwind,
            "gpu_launches": launches,
            "clocks": clock_info,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out), flush=True)
    for p in plans.values():
        p.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
