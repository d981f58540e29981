"""GPU: the C++ bssnrhs shim (reference signature, bssn:: globals) driven by a
small host program, against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po
from sympygr_b200 import build

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _driver(tmp_path):
    shim = build.build_shim()
    exe = str(tmp_path / "shim_test")
    subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(REPO, "sympygr_b200", "shim",
                                                             "shim_test_main.cpp"),
                    shim, "-Wl,-rpath," + os.path.dirname(shim), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("n,bflag,sigma,entry", [(17, 0x00, 0.2, "rhs"), (21, 0x3F, 0.35, "rhs"),
                                                (19, 0x15, 0.3, "sep"), (45, 0x2A, 0.25, "threads")])
def test_shim_matches_oracle(tmp_path, n, bflag, sigma, entry):
    exe = _driver(tmp_path)
    p0, h = -0.4, 0.8 / n
    u, blk = po.fake_block(n, (p0, p0, p0), h, bflag)
    inp, out = tmp_path / "u.bin", tmp_path / "r.bin"
    u.astype(np.float64).tofile(inp)
    # "threads": 4 host threads calling bssnrhs at once, each with the shim's per-thread
    # context, every result bitwise equal to the first call's
    extra = [entry] if entry in ("sep", "threads") else []
    subprocess.run([exe, str(inp), str(out), str(n), repr(p0), repr(h), str(bflag), repr(sigma),
                    *extra], check=True)
    got = np.fromfile(out, dtype=np.float64).reshape(24, -1)
    ref = po.oracle_rhs(u, blk, po.params(ko_sigma=sigma))
    mx, _ = po.rel_errors(po.interior(got, blk), po.interior(ref, blk))
    assert mx.max() < 1e-12


def test_shim_physical_constraints_matches_oracle(tmp_path):
    exe = _driver(tmp_path)
    n, p0, h, bflag = 19, -0.3, 0.04, 0x2A
    u, blk = po.fake_block(n, (p0, p0, p0), h, bflag)
    inp, out = tmp_path / "u.bin", tmp_path / "c.bin"
    u.astype(np.float64).tofile(inp)
    subprocess.run([exe, str(inp), str(out), str(n), repr(p0), repr(h), str(bflag), "0.1", "con"],
                   check=True)
    got = np.fromfile(out, dtype=np.float64).reshape(6, -1)
    ref = po.interior(po.oracle_constraints(u, blk), blk)
    mx, _ = po.rel_errors(po.interior(got[:4], blk), ref)
    assert mx.max() < 1e-12
    assert np.all(got[4:] == 0.0)  # the Psi4 arrays are left untouched
