"""CPU, world size 2 over gloo: the host logic `bench.py` runs under torchrun with N > 1.

Each rank evaluates its own seeded batch (weak scaling, no collective on the data path);
the timing is the maximum over ranks and the point count the sum over ranks.  Here each
rank evaluates its (small) batch through the oracle, standing in for the device work,
and the test checks the cross-rank reductions, that the ranks' batches differ, and that
`--impl reference` does its work on rank 0 only.  A second test has one rank raise
between steps: the other must leave its next reduction with an error, not wait.
"""
import datetime
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import bench
        from oracle import pyoracle as po
        from sympygr_b200 import workloads as wl

        blocks, total = wl.batch_blocks(sizes=(13, 16), counts=(3, 2), seed=rank)
        u = np.zeros((24, total))
        for b in blocks:
            x, y, z = wl.coords(b)
            u[:, b.offset:b.offset + b.npad] = po.fake_initial_data(x, y, z).reshape(24, -1)
        rhs = np.zeros_like(u)
        for b in blocks:
            po.oracle_rhs(u, b, po.params(ko_sigma=0.1), rhs=rhs)
        npts = sum(b.ninterior for b in blocks)
        ms = bench.max_over_ranks(5.0 + 2.0 * rank, dist, "cpu")
        tot = bench.sum_over_ranks(npts, dist, "cpu")
        checksum = float(np.abs(rhs).sum())
        ref = bench.reference_arm(type("A", (), {"warmup": 0, "steps": 1, "ref_fraction": 0.0})(),
                                  rank, world) if rank == 1 else None
        np.save(os.path.join(outdir, f"r{rank}.npy"),
                np.array([ms, tot, npts, checksum, 0.0 if ref is None else 1.0]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_bench(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                       start_method="spawn", join=True)
    r0, r1 = (np.load(tmp_path / f"r{r}.npy") for r in (0, 1))
    assert r0[0] == r1[0] == 7.0           # max over ranks, seen by every rank
    assert r0[1] == r1[1] == r0[2] + r1[2]  # points summed over ranks
    assert r0[3] != r1[3]                   # each rank evaluated its own batch
    assert r1[4] == 0.0                     # the reference arm runs on rank 0 only


def _failing_worker(rank, world, port, outdir, timeout_s):
    """Rank 1 raises between steps (no collective in flight); rank 0 must leave its next
    reduction with an error within the process-group timeout, not wait for good."""
    import time

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    import bench

    bench.max_over_ranks(1.0 + rank, dist, "cpu")  # one healthy step on both ranks
    if rank == 1:
        raise RuntimeError("planted failure on rank 1")
    t0 = time.monotonic()
    try:
        bench.max_over_ranks(3.0, dist, "cpu")
        status = "completed"
    except Exception as ex:  # gloo reports the lost peer or the timeout
        status = type(ex).__name__
    with open(os.path.join(outdir, "r0.txt"), "w") as f:
        f.write(f"{status} {time.monotonic() - t0:.2f}")


def test_a_failed_rank_ends_the_others_next_reduction_with_an_error(tmp_path):
    pytest.importorskip("torch")
    import torch.multiprocessing as mp

    timeout_s = 10
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, str(tmp_path), timeout_s))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
        p.join()
    assert not alive, "a rank waited past the process-group timeout"
    assert procs[1].exitcode != 0
    assert procs[0].exitcode == 0
    status, secs = (tmp_path / "r0.txt").read_text().split()
    assert status != "completed"
    assert float(secs) < timeout_s + 30
