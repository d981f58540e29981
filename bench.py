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
    python bench.py --profile-case {mixed,fp64} [--profile-steps N]   # small ncu case

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
MIXED_BAR = 1e-6

# Algorithmic work per interior point of the reference's algorithm (bssnrhs,
# bssn/src/rhs.cpp:80-388):
#  * the per-point algebra: 4137 operations after the reference's CSE
#    (bssn/src/bssneqs_eta_const_standard_gauge.cpp:1028);
#  * the stencils: 105 first derivatives (72 + 33 mixed) x 12, 33 diagonal second
#    derivatives x 14, 72 KO rows x 14, the KO add 24 x 4, eta damping ~10.
# FP64 path: all of it in FP64.  MIXED: the algebra in FP32, the stencils in FP64
# (their differences; the weighted sums of the split-precision rows run in FP32).
FLOPS_ALGEBRA = 4137
FLOPS_STENCIL = 105 * 12 + 33 * 14 + 72 * 14 + 24 * 4 + 10
# Bytes per interior point an evaluation must move at the least: the 24 state
# variables over the padded blocks (read) and the 24 right-hand sides (written).
BYTES_VARS = 24 * 8
# DRAM bytes per interior point of each kernel of an evaluation, from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of a 3.15M-point case of the batch's
# large blocks (four 69^3 and one 135^3, one flagged face): `python bench.py
# --profile-case {mixed,fp64} [--single-pass]` (derivative stage: its two kernels summed;
# the one-pass kernel with its default 128-slot ring).
NCU_TRAFFIC_PER_POINT = {"mixed": {"derivs": 375.0 + 646.0, "algebra": 1124.0, "single_pass": 836.0},
                         "fp64": {"derivs": 580.0 + 1083.0, "algebra": 1897.0}}
REF_STEP_CAP, REF_WARMUP_CAP = 3, 1  # reference arm: ~32 s per full-batch step on 16 threads

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
    """nvidia-smi clocks/throttle sampling during the timed region: started before the
    warm-up (nvidia-smi takes a moment to begin), every 100 ms, and only the samples
    taken between begin() and end() count (all of them if none fell there)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None
        self.window = (None, None)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def begin(self):
        self.window = (time.monotonic(), None)

    def end(self):
        self.window = (self.window[0], time.monotonic())

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
        t0, t1 = self.window
        inside = [ln for t, ln in self.lines if t0 is not None and t1 is not None and t0 <= t <= t1]
        lines = inside or [ln for _, ln in self.lines]
        sm, smax, reasons, power = [], None, set(), []
        for ln in lines:
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
                "reasons": sorted(reasons), "samples": len(sm), "in_timed_region": bool(inside),
                "power_w_max": max(power) if power else None}


def host_cpu() -> dict:
    """This host's CPU: model, logical CPUs, physical cores (distinct (package, core)
    pairs of /proc/cpuinfo; sockets x cores per socket from lscpu where that is absent)."""
    model, pairs, phys, core = None, set(), None, None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name" and model is None:
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif k == "" and phys is not None and core is not None:
                    pairs.add((phys, core))
                    phys = core = None
        if phys is not None and core is not None:
            pairs.add((phys, core))
    except OSError:
        pass
    physical = len(pairs) or None
    if physical is None:
        try:
            out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
            kv = dict(ln.split(":", 1) for ln in out.splitlines() if ":" in ln)
            physical = int(kv["Socket(s)"].strip()) * int(kv["Core(s) per socket"].strip())
        except Exception:
            physical = None
    return {"model": model, "logical": os.cpu_count() or 1, "physical_cores": physical}


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


def workload_config(nblocks: int, npts: int) -> dict:
    """The `config` object of both arms (identical, so the two lines compare)."""
    return {"workload": WORKLOAD, "blocks": nblocks, "interior_points_per_gpu": npts,
            "l2": "inputs (26.7 GB per state) larger than L2; no flush"}


def compact(u_src, blocks, device_to_host=True):
    """The given blocks' slices of a [24, N] array (numpy or torch), re-offset compactly
    into a host numpy array (block starts 32-element aligned); returns (u, blocks)."""
    import numpy as np

    from sympygr_b200 import workloads as wl

    out, off = [], 0
    for b in blocks:
        out.append(wl.Block(off, b.sz, b.bflag, b.pmin, b.pmax))
        off += ((b.npad + 31) // 32) * 32
    u = np.zeros((24, off))
    for b, o in zip(blocks, out):
        seg = u_src[:, b.offset:b.offset + b.npad]
        u[:, o.offset:o.offset + o.npad] = seg.cpu().numpy() if hasattr(seg, "cpu") else seg
    return u, out


def host_batch(blocks):
    """Host arrays for a block subset of the batch, re-offset compactly (block starts
    32-element aligned), filled with the two-puncture fields by numpy."""
    import numpy as np

    from sympygr_b200 import workloads as wl

    out, off = [], 0
    for b in blocks:
        out.append(wl.Block(off, b.sz, b.bflag, b.pmin, b.pmax))
        off += ((b.npad + 31) // 32) * 32
    u = np.zeros((24, off))
    punct = [(-4.0, 0.0, 0.0, 0.5), (4.0, 0.0, 0.0, 0.5)]
    for b in out:
        x, y, z = wl.coords(b)
        wl._bl_fields(u, slice(b.offset, b.offset + b.npad), x, y, z, punct)
    return u, out


def cpu_reference_run(u_host, blocks, nthreads, flavour="fast"):
    """The reference's own CPU bssnrhs (compiled from its sources) over a block list
    in its block-parallel OpenMP loop; returns (seconds, interior points, rhs)."""
    import numpy as np

    from oracle import pyoracle as po

    rhs = np.zeros_like(u_host)
    prm = po.params(ko_sigma=SIGMA)
    secs = po.ref_blocks_omp(u_host, rhs, blocks, prm, nthreads=nthreads, flavour=flavour)
    return secs, sum(b.ninterior for b in blocks), rhs


def reference_arm(args, rank, world):
    """`--impl reference`: the reference's CPU bssnrhs on this host's cores over the
    whole 3000-block batch (or the `--ref-fraction` class-proportional sample)."""
    if rank != 0:
        return None
    from oracle import pyoracle as po
    from sympygr_b200 import workloads as wl

    if not po.have_reference("fast"):
        return {"impl": "reference", "unavailable": "reference build oracle/_ref/libbssn_ref_fast*.so missing"}
    cpu = host_cpu()
    nthreads = cpu["logical"]
    frac = args.ref_fraction if 0 < args.ref_fraction < 1 else 1.0
    blocks, _ = wl.batch_blocks(seed=0)
    npts_all = sum(b.ninterior for b in blocks)
    sample = blocks if frac >= 1.0 else stratified_blocks(blocks, frac)
    # the batch's data on the host (the GPU arm's fields, computed with numpy)
    u, sblocks = host_batch(sample)
    # big blocks first so the block-parallel loop does not end on a long tail
    sblocks = sorted(sblocks, key=lambda b: -b.npad)
    warm = max(0, min(args.warmup, REF_WARMUP_CAP))
    steps = max(1, min(args.steps, REF_STEP_CAP))
    for _ in range(warm):
        cpu_reference_run(u, sblocks, nthreads)
    times, pts = [], 0
    for _ in range(steps):
        s, pts, _ = cpu_reference_run(u, sblocks, nthreads)
        times.append(s)
    t = statistics.median(times)
    val = pts / t / 1e6
    flav = os.path.basename(po.fast_flavour_path())
    sample_desc = ((f"the whole batch ({pts} interior points)" if frac >= 1.0 else
                    f"{len(sblocks)} of 3000 blocks ({frac:.3g} class-proportional sample, {pts} interior points)")
                   + f", largest blocks first, {nthreads} OpenMP threads over blocks; {flav}; "
                     f"median of {len(times)} steps after {warm} warm-up (capped at {REF_STEP_CAP} "
                     f"and {REF_WARMUP_CAP}: about 30 s per step)")
    return {
        "metric": METRIC, "value": round(val, 4), "unit": UNIT, "impl": "reference",
        "n_gpus": world, "steps": len(times), "warmup": warm,
        "ms_per_step": round(t * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(len(blocks), npts_all),
        "steps_cap": {"steps": REF_STEP_CAP, "warmup": REF_WARMUP_CAP,
                      "requested": {"steps": args.steps, "warmup": args.warmup}},
        "cpu_baseline": {"value": round(val, 4), "unit": UNIT, "cores": nthreads, "kind": "reference",
                         "physical_cores": cpu["physical_cores"], "cpu_model": cpu["model"],
                         "build": flav, "sample": sample_desc},
        "e2e": {"value": round(val, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def roofline(kernel, ms, npts, bytes_pp, f64_pp, f32_pp, hbm_peak, peak64, peak32, traffic_pp=None,
             launches=1, peak_src=""):
    """Roofline of one kernel (or a whole evaluation) from algorithmic work per point:
    `achieved`/`peak` against HBM (the contract's object), the FP64/FP32 pipe time
    beside it, and which roof binds (the longer of the two lower bounds)."""
    secs = ms * 1e-3
    gbs = bytes_pp * npts / secs / 1e9
    t_hbm = bytes_pp * npts / (hbm_peak * 1e9)
    # FP64 and FP32 arithmetic run on different pipes: the pipe bound is the longer one
    t_pipe = max(f64_pp * npts / (peak64 * 1e12), f32_pp * npts / (peak32 * 1e12))
    out = {"kernel": kernel, "bound": "hbm", "achieved": round(gbs, 1), "peak": hbm_peak, "unit": "GB/s",
           "frac": round(gbs / hbm_peak, 4),
           "traffic": None if traffic_pp is None else round(traffic_pp * npts / launches),
           "bytes_per_point": round(bytes_pp, 1), "launches_per_step": launches,
           "peak_source": peak_src,
           "pipe": {"fp64_flops_per_point": f64_pp, "fp32_flops_per_point": f32_pp,
                    "fp64_tflops": round(f64_pp * npts / secs / 1e12, 3),
                    "fp32_tflops": round(f32_pp * npts / secs / 1e12, 3),
                    "fp64_peak": round(peak64, 2), "fp32_peak": round(peak32, 2),
                    "frac": round(t_pipe / secs, 4),
                    "peak_source": "measured FMA-chain microbenchmark (b200bssn_fma_peak), this GPU"},
           "binding": "hbm" if t_hbm >= t_pipe else ("fp64 pipe" if f64_pp / peak64 >= f32_pp / peak32 else "fp32 pipe"),
           "frac_binding": round(max(t_hbm, t_pipe) / secs, 4)}
    if traffic_pp is not None:
        out["traffic_per_point"] = round(traffic_pp, 1)
        out["traffic_over_algorithmic"] = round(traffic_pp / bytes_pp, 2)
    return out


def profile_case(args):
    """Small case for ncu captures: four 69^3 blocks and one 135^3 block of the
    two-puncture batch, one with a flagged face (3.15M interior points, ~0.6 GB per
    state, larger than L2), evaluated twice with one plan; with --profile-steps also
    the constraint kernel once and that many RK4 steps."""
    import torch

    import sympygr_b200 as sg
    from sympygr_b200 import workloads as wl

    prec = sg.FP64 if args.profile_case == "fp64" else sg.MIXED
    # seed 5: one of the 69^3 blocks has a flagged face (8 % of the points), like the
    # 3000-block batch (about 10 % of its points lie in blocks with flagged faces)
    u, blocks = wl.two_puncture_batch_torch((69, 135), (4, 1), seed=5, device="cuda")
    rhs = torch.zeros_like(u)
    ctx = sg.Context(0)
    plan = sg.Plan(ctx, blocks, prec, single_pass=args.single_pass, ring_slots=args.ring_slots)
    prm = sg.Params.make(ko_sigma=SIGMA, precision=prec)
    for _ in range(2):
        plan.rhs_device(list(rhs), list(u), prm)
    plan.status()
    if args.profile_steps:
        norms = torch.zeros(len(blocks) * 8, dtype=torch.float64, device="cuda")
        plan.constraints_device(list(u), None, norms)
        rk = sg.RK4(plan)
        rk.init(list(u))
        for _ in range(args.profile_steps):
            rk.step(list(u), 1e-3, prm)
        torch.cuda.synchronize()
        rk.close()
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": args.profile_case, "single_pass": plan.single_pass, "points": plan.points,
                      "launches": plan.launches}))
    plan.close()
    ctx.close()


def single_block_rates(ctx, reps=5):
    """Mpoints/s of the two single-block configurations -- a 38^3 block of seeded
    sines on flat space and a 134^3 Brill-Lindquist block with all faces flagged --
    through the drop-in b200bssn_rhs (host arrays: copy in, evaluate, copy the
    interior out; the path the bssnrhs shim takes) and through a plan on device arrays,
    FP64 and MIXED.  Returns (rates, host inputs) -- the inputs feed the CPU baseline."""
    import numpy as np
    import torch

    import sympygr_b200 as sg
    from sympygr_b200 import workloads as wl

    out, inputs = {}, {}
    for name, (u, blk) in (("cfg1_38_sines", wl.flat_sines(38, 0.1, 0)),
                           ("cfg2_134_brill_lindquist", wl.brill_lindquist(134, 8.0, 1.0))):
        inputs[name] = (u, blk)
        rhs = np.zeros_like(u)
        ud = torch.from_numpy(u).cuda()
        rd = torch.zeros_like(ud)
        rec = {"interior_points": blk.ninterior}
        for prec, pname in ((sg.FP64, "fp64"), (sg.MIXED, "mixed")):
            prm = sg.Params.make(ko_sigma=SIGMA, precision=prec)
            # drop-in on host arrays (synchronous): wall clock around the calls
            sg.bssnrhs(ctx, list(rhs), list(u), blk.offset, blk.pmin, blk.pmax, blk.sz, blk.bflag, prm)
            t0 = time.perf_counter()
            for _ in range(reps):
                sg.bssnrhs(ctx, list(rhs), list(u), blk.offset, blk.pmin, blk.pmax, blk.sz, blk.bflag, prm)
            t_host = (time.perf_counter() - t0) / reps
            plan = sg.Plan(ctx, [blk], prec)
            stream = torch.cuda.ExternalStream(ctx.stream)
            for _ in range(3):
                plan.rhs_device(list(rd), list(ud), prm)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                plan.rhs_device(list(rd), list(ud), prm)
            e1.record(stream)
            e1.synchronize()
            t_dev = e0.elapsed_time(e1) * 1e-3 / reps
            plan.close()
            rec[pname] = {"dropin_host_mpts": round(blk.ninterior / t_host / 1e6, 2),
                          "dropin_host_ms": round(t_host * 1e3, 3),
                          "plan_device_mpts": round(blk.ninterior / t_dev / 1e6, 2),
                          "plan_device_ms": round(t_dev * 1e3, 3)}
        out[name] = rec
        del ud, rd
    return out, inputs


def cpu_baseline_leg(u_dev, blocks, rhs64_dev, single_inputs, ref_frac):
    """The reference's own CPU bssnrhs (timing build) on this host's cores: over a
    bounded class-proportional sample of the batch (the inputs copied from the GPU
    arm's device arrays) and on the two single-block configurations.  Also the FP64
    GPU path against the reference's parity build (-ffp-contract=off) on one block of
    each size class of that sample (flagged faces where the class has them)."""
    import numpy as np

    from oracle import pyoracle as po

    if not po.have_reference("fast"):
        return None, None
    cpu = host_cpu()
    nthreads = cpu["logical"]
    sample = stratified_blocks(blocks, ref_frac)
    uh, sb = compact(u_dev, sample)
    order = sorted(range(len(sb)), key=lambda i: -sb[i].npad)
    secs, pts, _ = cpu_reference_run(uh, [sb[i] for i in order], nthreads)
    flav = os.path.basename(po.fast_flavour_path())
    per_config = {"cfg3_batch_sample": {"mpts": round(pts / secs / 1e6, 4), "seconds": round(secs, 2),
                                        "interior_points": pts, "threads": nthreads}}
    for name, (u, blk) in single_inputs.items():
        # the reference parallelises over blocks only: one block runs on one thread
        s, p, _ = cpu_reference_run(u, [blk], nthreads)
        per_config[name] = {"mpts": round(p / s / 1e6, 4), "seconds": round(s, 2), "interior_points": p,
                            "threads": 1}
    cpu_rec = {"value": per_config["cfg3_batch_sample"]["mpts"], "unit": UNIT, "cores": nthreads,
               "kind": "reference", "physical_cores": cpu["physical_cores"], "cpu_model": cpu["model"],
               "build": flav,
               "sample": f"{len(sb)} blocks ({ref_frac:.3g} class-proportional sample of the batch, "
                         f"{pts} interior points, largest first), one pass, {secs:.2f} s, "
                         f"{nthreads} OpenMP threads over blocks",
               "per_config": per_config}
    # FP64 GPU vs the reference (parity build) on one block per class of the sample
    chk = []
    for n in sorted({b.sz[0] for b in blocks}):
        cls = [b for b in blocks if b.sz[0] == n]
        flagged = [b for b in cls if b.bflag]
        chk.append(flagged[0] if flagged else cls[0])
    uc, cb = compact(u_dev, chk)
    _, _, ref = cpu_reference_run(uc, cb, nthreads, flavour="parity")
    got, _ = compact(rhs64_dev, chk)
    worst, per_block = 0.0, []
    for b in cb:
        mx, _ = po.rel_errors(po.interior(got, b), po.interior(ref, b))
        nz = np.abs(po.interior(ref, b)).max(axis=1) > 0
        e = float(mx[nz].max()) if nz.any() else 0.0
        worst = max(worst, e)
        per_block.append({"n": b.sz[0], "bflag": b.bflag, "max_rel_err": float(f"{e:.3g}")})
    fp64_check = {"max_rel_err": worst, "bar": 1e-12, "blocks": per_block,
                  "against": "the reference's bssnrhs, parity build (-O2 -ffp-contract=off)"}
    return cpu_rec, fp64_check


def e2e_leg(ctx, blocks, u, args, dist, world):
    """The metric end to end through the host API (b200bssn_rhs_plan_host: H2D of the
    state, evaluate, D2H of the RHS, pinned host arrays), MIXED and FP64.  Each rank pins
    a state and an RHS copy of its batch; where the ranks on this node would need more
    than 60 % of its available memory, each times a class-proportional sample."""
    import torch

    import sympygr_b200 as sg
    from sympygr_b200 import workloads as wl

    local = max(1, _env_int("LOCAL_WORLD_SIZE", world))
    span = max(b.offset + b.npad for b in blocks)
    need = 2 * 24 * span * 8
    budget = int(0.6 * host_bytes_available() / local)
    hblocks, sample_note = blocks, None
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
    return u_h, hblocks, span, sample_note


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
    ap.add_argument("--no-single", action="store_true", help="skip the single-block configurations")
    ap.add_argument("--ref-fraction", type=float, default=0.0,
                    help="reference arm: class-proportional sample of the batch (0 or >= 1: the whole "
                         "batch); GPU arm's CPU-baseline leg: its sample (0: enough 135^3 blocks to "
                         "give every host core one, min 0.1)")
    ap.add_argument("--chunk-points", type=int, default=0)
    ap.add_argument("--slab-depth", type=int, default=0)
    ap.add_argument("--deriv-ctas", type=int, default=0, help="derivative CTAs per SM (0: max)")
    ap.add_argument("--single-pass", action="store_true",
                    help="MIXED headline on the one-pass kernel instead of the two-pass kernels")
    ap.add_argument("--ring-slots", type=int, default=0, help="one-pass ring slots (0: default)")
    ap.add_argument("--no-other", action="store_true", help="skip timing the other MIXED kernel set")
    ap.add_argument("--profile-case", choices=["mixed", "fp64"], default=None,
                    help="run the small ncu profiling case instead of the benchmark")
    ap.add_argument("--profile-steps", type=int, default=0)
    args = ap.parse_args()

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        out = reference_arm(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if args.profile_case:
        profile_case(args)
        return

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
    plans = {p: sg.Plan(ctx, blocks, p, args.chunk_points, args.slab_depth, args.deriv_ctas,
                        single_pass=args.single_pass, ring_slots=args.ring_slots)
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

    clocks = ClockSampler(local_rank)
    clocks.start()
    for prec in (sg.MIXED, sg.FP64):
        for _ in range(args.warmup):
            plans[prec].rhs_device(R, U, params[prec])
    torch.cuda.synchronize()

    clocks.begin()
    ms_mixed = timed(sg.MIXED, args.steps)
    clocks.end()
    clock_info = clocks.stop()
    ms_fp64 = timed(sg.FP64, args.steps)
    for p in plans.values():
        p.status()  # a bounded device wait that ran out would leave results incomplete

    # the other MIXED kernel set on the same batch: the two-pass kernels (derivative
    # scratch through HBM) or the one-pass kernel, whichever the headline did not use
    mixed_other = None
    if not args.no_other:
        other_single = not plans[sg.MIXED].single_pass
        p2 = sg.Plan(ctx, blocks, sg.MIXED, args.chunk_points, args.slab_depth, args.deriv_ctas,
                     single_pass=other_single, ring_slots=args.ring_slots)
        for _ in range(args.warmup):
            p2.rhs_device(R, U, params[sg.MIXED])
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            p2.rhs_device(R, U, params[sg.MIXED])
        e1.record(stream)
        e1.synchronize()
        ms2 = max_over_ranks(e0.elapsed_time(e1), dist) / args.steps
        d2, a2 = p2.profile(R, U, params[sg.MIXED])
        p2.status()
        p2.close()
        mixed_other = {"kernels": "one-pass" if other_single else "two-pass",
                       "value": round(sum_over_ranks(npts, dist) / (ms2 * 1e-3) / 1e6, 3),
                       "ms_per_step": round(ms2, 3), "deriv_ms": round(d2, 3), "algebra_ms": round(a2, 3)}

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

    # per-kernel device time of one evaluation (events between launches)
    prof = {}
    for prec in (sg.MIXED, sg.FP64):
        prof[prec] = plans[prec].profile(R, U, params[prec])
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

    padded = sum(b.npad for b in blocks)
    read_state = BYTES_VARS * padded / npts
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            hbm_peak = float(json.load(fh)["hbm_gbs"])
        peak_src = "measured (hbm_gbs of the measured-peaks file, copy test)"
    except Exception:
        hbm_peak, peak_src = 6650.0, "fallback 6.65 TB/s"
    rl = {}
    for prec, mode in ((sg.MIXED, "mixed"), (sg.FP64, "fp64")):
        d_ms, a_ms = prof[prec]
        tr = NCU_TRAFFIC_PER_POINT[mode]
        f32_alg = FLOPS_ALGEBRA if mode == "mixed" else 0
        f64_alg = 0 if mode == "mixed" else FLOPS_ALGEBRA
        if plans[prec].single_pass:
            # one kernel per evaluation: its roofline is the evaluation's
            one = roofline("bssn_fused_kernel<0> (one-pass: derivatives, algebra, KO, Sommerfeld)",
                           d_ms, npts, read_state + BYTES_VARS, FLOPS_STENCIL, f32_alg, hbm_peak, peak64,
                           peak32, tr.get("single_pass"), 1, peak_src)
            ev = roofline(f"whole {mode} evaluation (all launches)", ms_mixed if mode == "mixed" else ms_fp64,
                          npts, read_state + BYTES_VARS, FLOPS_STENCIL + f64_alg, f32_alg, hbm_peak, peak64,
                          peak32, tr.get("single_pass"), 1, peak_src)
            rl[mode] = {"single_pass": one, "evaluation": ev}
            continue
        nchunks = max(1, plans[prec].launches // 3)  # 3 launches per chunk
        rl[mode] = {
            # derivative stage: reads the state over the padded blocks; its scratch is
            # not algorithmic (the reference's algorithm needs no scratch traffic)
            "derivs": roofline(f"bssn_derivs_kind_kernel<{'float' if mode == 'mixed' else 'double'},*> (both kinds)",
                               d_ms, npts, read_state, FLOPS_STENCIL, 0, hbm_peak, peak64, peak32,
                               tr["derivs"], nchunks, peak_src),
            # algebra: the state at the point in, the 24 right-hand sides out
            "algebra": roofline(f"bssn_algebra_staged_kernel<{'float' if mode == 'mixed' else 'double'},0>",
                                a_ms, npts, 2 * BYTES_VARS, f64_alg, f32_alg, hbm_peak, peak64, peak32,
                                tr["algebra"], nchunks, peak_src),
            "evaluation": roofline(f"whole {mode} evaluation (all launches)",
                                   ms_mixed if mode == "mixed" else ms_fp64, npts,
                                   read_state + BYTES_VARS, FLOPS_STENCIL + f64_alg, f32_alg,
                                   hbm_peak, peak64, peak32, tr["derivs"] + tr["algebra"], 1, peak_src),
        }

    # the single-block configurations and the end-to-end legs run after the batch's
    # device timing; the RHS of the FP64 path is kept for the reference check
    single, single_inputs = (None, {})
    if not args.no_single:
        single, single_inputs = single_block_rates(ctx)

    cpu, fp64_check = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            frac = args.ref_fraction if args.ref_fraction > 0 else max(0.1, min(1.0, (os.cpu_count() or 1) / 30.0))
            cpu, fp64_check = cpu_baseline_leg(u, blocks, ref64, single_inputs, frac)
        except Exception as ex:  # the baseline is informational; never fail the bench on it
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {ex}"}
    del ref64

    e2e = None
    if not args.no_e2e:
        u_h, hblocks, span, sample_note = e2e_leg(ctx, blocks, u, args, dist, world)
        del rhs, u
        U = R = None
        torch.cuda.empty_cache()
        e2e_pts = sum_over_ranks(sum(b.ninterior for b in hblocks), dist)
        r_h = torch.empty(tuple(u_h.shape), dtype=u_h.dtype, pin_memory=True)
        UH, RH = [t.data_ptr() for t in u_h], [t.data_ptr() for t in r_h]
        nbytes = 24 * span * 8
        res = {}
        # MIXED and FP64 with the RHS ghosts zeroed, and MIXED with them left as the caller
        # had them (the reference's semantics: only the interiors come back)
        for prec, name, policy in ((sg.MIXED, "mixed", sg.GHOSTS_ZERO), (sg.FP64, "fp64", sg.GHOSTS_ZERO),
                                   (sg.MIXED, "preserve", sg.GHOSTS_PRESERVE)):
            hplan = plans[prec] if sample_note is None else sg.Plan(ctx, hblocks, prec, args.chunk_points,
                                                                     args.slab_depth, args.deriv_ctas)
            p_host = sg.Params.make(ko_sigma=SIGMA, precision=prec, ghost_policy=policy)
            hplan.rhs_host(RH, UH, span, p_host)  # warm-up (allocates staging)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.e2e_steps):
                hplan.rhs_host(RH, UH, span, p_host)
            e1.record(stream)
            e1.synchronize()
            res[name] = max_over_ranks(e0.elapsed_time(e1) / args.e2e_steps, dist)
            if sample_note is not None:
                hplan.close()
        # the transfer bound: both directions' bytes at the concurrent copy rate
        gbs = duplex_copy_gbs(u_h, r_h)
        copy_ms = max_over_ranks(nbytes / (gbs * 1e9) * 1e3, dist)
        del u_h, r_h
        ms = res["mixed"]
        e2e = {"value": round(e2e_pts / (ms * 1e-3) / 1e6, 3), "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "ms_per_step": round(ms, 2), "steps": args.e2e_steps,
               "api": "b200bssn_rhs_plan_host (pinned host arrays, ghosts zeroed), MIXED",
               "sample": sample_note,
               "fp64": {"value": round(e2e_pts / (res["fp64"] * 1e-3) / 1e6, 3),
                        "ms_per_step": round(res["fp64"], 2)},
               "preserve": {"value": round(e2e_pts / (res["preserve"] * 1e-3) / 1e6, 3),
                            "ms_per_step": round(res["preserve"], 2),
                            "api": "the same, MIXED, ghosts left as the caller had them (the "
                                   "interiors come back; no RHS upload)"},
               "copy_bound": {"duplex_gbs_per_direction": round(gbs, 1),
                              "ms_per_step": round(copy_ms, 2),
                              "value": round(e2e_pts / (copy_ms * 1e-3) / 1e6, 3),
                              "frac": round(copy_ms / ms, 4),
                              "how": "1 GiB H2D and D2H copies at once from/to the same pinned "
                                     "arrays, one stream each; bytes per step / that rate"}}

    if rank == 0:
        d_ms, a_ms = prof[sg.MIXED]
        d64, a64 = prof[sg.FP64]
        out = {
            "metric": METRIC, "value": round(val_mixed, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_mixed, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 state+stencils / f32 algebra", "data": "synthetic",
            "config": workload_config(len(blocks), npts) if args.scale == 1.0 else
            dict(workload_config(len(blocks), npts), scale=args.scale),
            "fp64": {"value": round(val_fp64, 3), "ms_per_step": round(ms_fp64, 3),
                     "deriv_ms": round(d64, 3), "algebra_ms": round(a64, 3),
                     "vs_reference": fp64_check},
            "mixed_kernels": "one-pass" if plans[sg.MIXED].single_pass else "two-pass",
            "mixed_other_kernels": mixed_other,
            "mixed_vs_fp64": {"speedup": round(val_mixed / val_fp64, 3),
                              "max_rel_err": mixed_max_rel, "bar": MIXED_BAR,
                              "per_var_max_rel": [float(f"{x:.3g}") for x in per_var_max],
                              "per_var_rms_rel": [float(f"{x:.3g}") for x in per_var_rms]},
            "kernels_ms": ({"single_pass": round(d_ms, 3)} if plans[sg.MIXED].single_pass
                           else {"deriv": round(d_ms, 3), "algebra": round(a_ms, 3)}),
            # dominant kernel of the headline (mixed) evaluation: the one-pass kernel (or,
            # on the two-pass kernels, the derivative stage)
            "roofline": rl["mixed"]["single_pass"] if plans[sg.MIXED].single_pass else rl["mixed"]["derivs"],
            "roofline_algebra": rl["mixed"].get("algebra"),
            "roofline_evaluation": rl["mixed"]["evaluation"],
            "roofline_fp64": rl["fp64"],
            "single_block": single,
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
