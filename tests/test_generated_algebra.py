"""CPU check of the generated device algebra: the staged CUDA template, compiled
for the host with RT=double, against the oracle's flat C algebra (which is pinned
to the reference's bssneqs_eta_const_standard_gauge.cpp through the golden tests)
at seeded random points.  Catches printer and generator mistakes without a GPU."""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def algcheck(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("alg") / "algcheck")
    subprocess.run(["g++", "-O1", "-std=c++17", os.path.join(HERE, "algebra_host_check.cpp"),
                    "-x", "c", os.path.join(REPO, "oracle", "bssn_oracle_algebra.c"),
                    os.path.join(REPO, "oracle", "bssn_oracle_constraints.c"),
                    os.path.join(REPO, "oracle", "bssn_oracle_algebra_adv.c"), "-x", "none",
                    "-I", os.path.join(REPO, "sympygr_b200", "csrc", "generated"),
                    "-I", os.path.join(REPO, "oracle"), "-o", exe, "-lm"], check=True)
    return exe


def test_staged_device_algebra_matches_oracle(algcheck):
    out = subprocess.run([algcheck, "3000"], capture_output=True, text=True, check=True).stdout
    rel = np.array([float(l.split()[1]) for l in out.strip().splitlines()])
    assert rel.shape == (24,)
    assert rel.max() < 1e-13, rel


def test_staged_constraint_algebra_matches_oracle(algcheck):
    """The staged device constraint template (ham, mom0..2) against the oracle's flat
    C constraints, which tests/test_oracle.py pins to the reference's own
    physical_constraints."""
    out = subprocess.run([algcheck, "3000", "con"], capture_output=True, text=True,
                         check=True).stdout
    rel = np.array([float(l.split()[1]) for l in out.strip().splitlines()])
    assert rel.shape == (4,)
    assert rel.max() < 1e-13, rel


def test_staged_upwind_algebra_matches_oracle(algcheck):
    """The upwind-mode device template (advective derivatives in slots 138..209) against
    the oracle's flat C twin."""
    out = subprocess.run([algcheck, "3000", "adv"], capture_output=True, text=True,
                         check=True).stdout
    rel = np.array([float(l.split()[1]) for l in out.strip().splitlines()])
    assert rel.shape == (24,)
    assert rel.max() < 1e-13, rel


def test_upwind_algebra_reduces_to_the_reference_algebra(algcheck):
    """Fed the centred first derivatives in its advective slots, the upwind-mode algebra
    is the reference's algebra (the oracle's, pinned to the reference)."""
    out = subprocess.run([algcheck, "3000", "advsame"], capture_output=True, text=True,
                         check=True).stdout
    rel = np.array([float(l.split()[1]) for l in out.strip().splitlines()])
    assert rel.max() < 1e-13, rel


def test_split_algebra_matches_oracle(algcheck):
    """The two-part FP64 algebra (the six At_rhs with the Ricci tensor, then the other 18
    outputs, each part pruned to the stages it needs and CSE'd on its own) against the
    oracle's flat C algebra; every output is written by one of the parts."""
    out = subprocess.run([algcheck, "3000", "split"], capture_output=True, text=True,
                         check=True).stdout
    rel = np.array([float(l.split()[1]) for l in out.strip().splitlines()])
    assert rel.shape == (24,)
    assert np.isfinite(rel).all() and rel.max() < 1e-13, rel
