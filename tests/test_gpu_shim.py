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


@pytest.mark.parametrize("n,bflag,sigma", [(17, 0x00, 0.2), (21, 0x3F, 0.35)])
def test_shim_matches_oracle(tmp_path, n, bflag, sigma):
    shim = build.build_shim()
    exe = str(tmp_path / "shim_test")
    subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(REPO, "sympygr_b200", "shim",
                                                             "shim_test_main.cpp"),
                    shim, "-Wl,-rpath," + os.path.dirname(shim), "-o", exe], check=True)
    p0, h = -0.4, 0.8 / n
    u, blk = po.fake_block(n, (p0, p0, p0), h, bflag)
    inp, out = tmp_path / "u.bin", tmp_path / "r.bin"
    u.astype(np.float64).tofile(inp)
    subprocess.run([exe, str(inp), str(out), str(n), repr(p0), repr(h), str(bflag), repr(sigma)],
                   check=True)
    got = np.fromfile(out, dtype=np.float64).reshape(24, -1)
    ref = po.oracle_rhs(u, blk, po.params(ko_sigma=sigma))
    mx, _ = po.rel_errors(po.interior(got, blk), po.interior(ref, blk))
    assert mx.max() < 1e-12
