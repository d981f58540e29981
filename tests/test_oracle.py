"""CPU tests of the oracle: the C restatement against the reference's own outputs
(golden fixtures made by tests/golden/make_golden.py from the reference build) and,
where the reference build is present, against the reference directly."""
import glob
import hashlib
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from sympygr_b200 import workloads as wl

TOL = 1e-12  # norm-wise relative, per variable


def _sha(u):
    return hashlib.sha256(np.ascontiguousarray(u, dtype=np.float64).tobytes()).hexdigest()


def _fake_cases(golden_dir):
    return sorted(glob.glob(os.path.join(golden_dir, "fake_*.npz")))


def test_golden_files_present(golden_dir):
    assert len(_fake_cases(golden_dir)) >= 4
    for name in ("sines_38.npz", "bl_134.npz"):
        assert os.path.exists(os.path.join(golden_dir, name))


@pytest.mark.parametrize("case", ["fake_13_b00", "fake_13_b3f", "fake_13_b05", "fake_17_b2a"])
def test_oracle_matches_reference_golden_fake(golden_dir, oracle_lib, case):
    g = np.load(os.path.join(golden_dir, case + ".npz"))
    u, blk = po.fake_block(int(g["n"]), tuple(g["pmin"]), float(g["h"]), int(g["bflag"]))
    assert _sha(u) == str(g["input_sha"]), "fake_initial_data restatement drifted"
    r = po.oracle_rhs(u, blk, po.params(ko_sigma=float(g["sigma"])))
    mx, rms = po.rel_errors(po.interior(r, blk), g["rhs_interior"])
    assert mx.max() < TOL, (mx.max(), int(np.argmax(mx)))


@pytest.mark.parametrize("name,maker", [("sines_38", lambda: wl.flat_sines(38, 0.1, 0))])
def test_oracle_matches_reference_golden_cfg1(golden_dir, oracle_lib, name, maker):
    g = np.load(os.path.join(golden_dir, name + ".npz"))
    u, blk = maker()
    assert _sha(u) == str(g["input_sha"])
    r = po.interior(po.oracle_rhs(u, blk, po.params(ko_sigma=float(g["sigma"]))), blk)
    ref = g["sample_rhs"]
    got = r[:, g["sample_index"]]
    scale = np.abs(g["checksums"][:, 2])[:, None]
    assert (np.abs(got - ref) / scale).max() < TOL
    cs = g["checksums"]
    assert np.allclose(np.abs(r).max(axis=1), cs[:, 2], rtol=1e-12, atol=0)
    assert np.allclose((r ** 2).sum(axis=1), cs[:, 1], rtol=1e-10, atol=0)


def test_workload_inputs_stable(golden_dir):
    g = np.load(os.path.join(golden_dir, "bl_134.npz"))
    u, blk = wl.brill_lindquist(134, 8.0, 1.0)
    assert _sha(u) == str(g["input_sha"])
    assert blk.bflag == int(g["bflag"]) == 0x3F


@pytest.mark.skipif(not po.have_reference("parity"), reason="reference build not present")
@pytest.mark.parametrize("n,bflag", [(13, 0), (13, 0x3F), (15, 0x11), (21, 0x22), (16, 0x0C)])
def test_oracle_vs_reference_direct(oracle_lib, n, bflag):
    u, blk = po.fake_block(n, (-0.4, 0.25, -0.15), 0.06, bflag)
    prm = po.params(ko_sigma=0.3, eta_r0=0.2, eta_damping_exp=2.0)  # exercise eta damping
    a = po.oracle_rhs(u, blk, prm)
    b = po.ref_rhs(u, blk, prm)
    mx, _ = po.rel_errors(po.interior(a, blk), po.interior(b, blk))
    assert mx.max() < TOL
    # ghost points of the RHS are untouched by both
    mask = ~wl.interior_mask(blk).ravel()
    assert np.all(a[:, mask] == 0) and np.all(b[:, mask] == 0)


@pytest.mark.skipif(not po.have_reference("parity"), reason="reference build not present")
@pytest.mark.parametrize("n,bflag", [(13, 0), (17, 0x3F), (21, 0x15)])
def test_reference_staged_variant_equals_oracle(oracle_lib, n, bflag):
    """bssnrhs_sep (bssn/src/rhs.cpp:392-825, the BSSN_RHS_STAGED_COMP build) computes the
    same right-hand side as bssnrhs, so one path serves both entry points."""
    u, blk = po.fake_block(n, (-0.45, 0.2, -0.3), 0.9 / n, bflag)
    prm = po.params(ko_sigma=0.3)
    a = po.interior(po.oracle_rhs(u, blk, prm), blk)
    b = po.interior(po.ref_rhs_sep(u, blk, prm), blk)
    mx, _ = po.rel_errors(a, b)
    assert mx.max() < TOL


def test_ghost_insensitive_with_all_faces(oracle_lib):
    """With every face flagged, one-sided closures never read the ghost layer."""
    u, blk = po.fake_block(15, (-0.4, 0.25, -0.15), 0.06, 0x3F)
    a = po.interior(po.oracle_rhs(u, blk, po.params(ko_sigma=0.2)), blk)
    u2 = u.copy()
    mask = ~wl.interior_mask(blk).ravel()
    u2[:, mask] += np.random.default_rng(3).normal(size=(24, mask.sum()))
    b = po.interior(po.oracle_rhs(u2, blk, po.params(ko_sigma=0.2)), blk)
    assert np.array_equal(a, b)


def _poly_block(n, deg, axis, bflag):
    blk = wl.Block(0, (n, n, n), bflag, (-1.0, -0.5, -0.75), (-1.0 + (n - 1) * 0.1,
                   -0.5 + (n - 1) * 0.1, -0.75 + (n - 1) * 0.1))
    x, y, z = wl.coords(blk)
    c = (x, y, z)[axis]
    return blk, c, c ** deg


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_stencils_exact_on_polynomials(oracle_lib, axis):
    """Centred first/second derivatives are exact for degree <= 6 polynomials, the
    4th-order closures for degree <= 4; KO annihilates degree <= 5."""
    import ctypes

    lib = oracle_lib
    n = 17
    fns = {0: ("bssn_oracle_deriv64_x", "bssn_oracle_deriv64_xx", "bssn_oracle_ko_deriv42_x"),
           1: ("bssn_oracle_deriv64_y", "bssn_oracle_deriv64_yy", "bssn_oracle_ko_deriv42_y"),
           2: ("bssn_oracle_deriv64_z", "bssn_oracle_deriv64_zz", "bssn_oracle_ko_deriv42_z")}[axis]
    for bflag, deg in [(0, 6), (0x3F, 4)]:
        blk, c, f = _poly_block(n, deg, axis, bflag)
        f = np.ascontiguousarray(f.ravel())
        sz = (ctypes.c_uint * 3)(n, n, n)
        inner = wl.interior_mask(blk).ravel()
        for name, expect, tol in [(fns[0], deg * c.ravel() ** (deg - 1), 1e-8),
                                  (fns[1], deg * (deg - 1) * c.ravel() ** (deg - 2), 1e-6)]:
            out = np.zeros_like(f)
            getattr(lib, name)(out.ctypes.data_as(ctypes.c_void_p), f.ctypes.data_as(ctypes.c_void_p),
                               ctypes.c_double(0.1), sz, ctypes.c_uint(bflag))
            err = np.abs(out[inner] - expect[inner]).max() / np.abs(expect[inner]).max()
            assert err < tol, (name, bflag, err)
        blk, c, f = _poly_block(n, 5, axis, 0)
        f = np.ascontiguousarray(f.ravel())
        out = np.zeros_like(f)
        getattr(lib, fns[2])(out.ctypes.data_as(ctypes.c_void_p), f.ctypes.data_as(ctypes.c_void_p),
                             ctypes.c_double(0.1), sz, ctypes.c_uint(0))
        assert np.abs(out[inner]).max() < 1e-9


# ---- Hamiltonian and momentum constraints ----------------------------------------

@pytest.mark.parametrize("case", ["con_fake_13_b00", "con_fake_17_b2a"])
def test_oracle_constraints_match_reference_golden(golden_dir, oracle_lib, case):
    """The C restatement of the constraints against the reference's own
    physical_constraints (bssn/CodeGen/physcon.cpp:12) on fake_initial_data."""
    g = np.load(os.path.join(golden_dir, case + ".npz"))
    u, blk = po.fake_block(int(g["n"]), tuple(g["pmin"]), float(g["h"]), int(g["bflag"]))
    assert _sha(u) == str(g["input_sha"])
    c = po.interior(po.oracle_constraints(u, blk), blk)
    mx, _ = po.rel_errors(c, g["con_interior"])
    assert mx.max() < TOL, mx


def test_oracle_constraints_match_reference_golden_bl(golden_dir, oracle_lib):
    g = np.load(os.path.join(golden_dir, "con_bl_70.npz"))
    u, blk = wl.brill_lindquist(70, 8.0, 1.0)
    assert _sha(u) == str(g["input_sha"])
    c = po.interior(po.oracle_constraints(u, blk), blk)
    scale = np.maximum(g["checksums"][:, 2], 1e-300)[:, None]  # momentum is exactly 0 here
    assert (np.abs(c[:, g["sample_index"]] - g["sample_con"]) / scale).max() < TOL
    assert np.allclose(np.abs(c).max(axis=1), g["checksums"][:, 2], rtol=1e-12, atol=0)


@pytest.mark.skipif(not po.have_reference("parity"), reason="reference build not present")
@pytest.mark.parametrize("n,bflag", [(13, 0x3F), (16, 0x15), (19, 0x2A)])
def test_oracle_constraints_vs_reference_direct(oracle_lib, n, bflag):
    u, blk = po.fake_block(n, (-0.4, 0.25, -0.15), 0.06, bflag)
    a = po.interior(po.oracle_constraints(u, blk), blk)
    b = po.interior(po.ref_constraints(u, blk), blk)[:4]
    mx, _ = po.rel_errors(a, b)
    assert mx.max() < TOL, mx


def test_constraints_vanish_for_exact_solution(oracle_lib):
    """Brill-Lindquist data (conformally flat, K = A = 0, Gt = 0) solve the
    Hamiltonian and momentum constraints: the discrete residual is truncation error
    that shrinks at the stencils' order as h -> 0."""
    res = []
    for n in (38, 70):
        u, blk = wl.brill_lindquist(n, 8.0, 1.0)
        c = po.interior(po.oracle_constraints(u, blk), blk)
        # away from the puncture, where the fields are smooth on both grids
        x, y, z = (a.ravel() for a in wl.coords(blk))
        r = np.sqrt(x ** 2 + y ** 2 + z ** 2)[wl.interior_mask(blk).ravel()]
        far = (r > 3.0) & (r < 6.0)
        assert np.all(c[1:] == 0.0)  # momentum: every term carries A, K or grad K
        res.append(np.abs(c[0, far]).max())
    assert res[1] < res[0] / 8.0, res


# ---- RK4 time stepping -------------------------------------------------------------

def test_oracle_rk4_is_fourth_order():
    """Step doubling: one step of dt against two of dt/2 differ by the local error,
    O(dt^5), so halving dt shrinks the difference ~32x."""
    u0, blk = po.fake_block(15, (-0.4, 0.25, -0.15), 0.06, 0x3F)
    prm = po.params(ko_sigma=0.1)
    mask = po.interior_elements([blk], u0.shape[1])

    def run(dt, n):
        u = u0.copy()
        rk = po.OracleRK4([blk], u.shape[1], prm)
        rk.init(u)
        for _ in range(n):
            rk.step(u, dt)
        assert np.array_equal(u[:, ~mask], u0[:, ~mask])  # ghosts never written
        return u[:, mask]

    d = []
    for dt in (1e-3, 5e-4):
        a, b = run(dt, 1), run(dt / 2, 2)
        d.append((np.abs(a - b).max(axis=1) / np.abs(a).max(axis=1)).max())
    assert 20.0 < d[0] / d[1] < 40.0, d


# ---- opt-in upwind mode: 4th-order upwind advective derivatives --------------------

def test_oracle_upwind_derivatives_match_reference_golden(golden_dir, oracle_lib):
    """The oracle's deriv42adv restatement against the reference's own deriv42adv_{x,y,z}
    outputs (bitwise: same coefficients and summation order, no FMA contraction)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(golden_dir, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g = np.load(os.path.join(golden_dir, "adv42.npz"))
    f, beta, sz = mg.adv_inputs()
    assert _sha(np.concatenate([f, beta])) == str(g["input_sha"])
    for axis in range(3):
        for bflag in (0x00, 0x3F):
            got = po.oracle_deriv42adv(axis, f, float(g["h"]), sz, beta, bflag)
            assert np.array_equal(got, g[f"d{axis}_b{bflag:02x}"]), (axis, bflag)


@pytest.mark.skipif(not po.have_reference("parity"), reason="reference build not present")
@pytest.mark.parametrize("axis", [0, 1, 2])
def test_oracle_upwind_derivatives_vs_reference_direct(oracle_lib, axis):
    rng = np.random.default_rng(axis)
    sz = (14, 13, 16)
    f = rng.standard_normal(sz[0] * sz[1] * sz[2])
    beta = rng.standard_normal(f.size)
    for bflag in (0x00, 0x3F, 1 << (2 * axis), 2 << (2 * axis), 0x15, 0x2A):
        a = po.oracle_deriv42adv(axis, f, 0.05, sz, beta, bflag)
        b = po.ref_deriv42adv(axis, f, 0.05, sz, beta, bflag)
        assert np.array_equal(a, b), bflag


def test_oracle_upwind_rhs_differs_only_in_advection(oracle_lib):
    """With zero shift every advective term vanishes, so the upwind-mode RHS equals the
    standard RHS; with a shift they differ (by the advection terms only)."""
    u, blk = po.fake_block(15, (-0.4, 0.25, -0.15), 0.06, 0x15)
    prm = po.params(ko_sigma=0.2)
    base = po.interior(po.oracle_rhs(u, blk, prm), blk)
    adv = po.interior(po.oracle_rhs_adv(u, blk, prm), blk)
    assert not np.allclose(adv, base)
    u0 = u.copy()
    u0[6:9] = 0.0  # beta0..2
    a = po.interior(po.oracle_rhs(u0, blk, prm), blk)
    b = po.interior(po.oracle_rhs_adv(u0, blk, prm), blk)
    mx, _ = po.rel_errors(b, a)
    assert mx.max() < 1e-13


def test_oracle_is_clean_under_address_and_undefined_behaviour_sanitizers(tmp_path):
    """The oracle's C (stencils, closures, upwind rows, algebra, constraints) built with
    -fsanitize=address,undefined and run on one block with every face-flag pattern."""
    import subprocess

    here = os.path.dirname(os.path.abspath(__file__))
    orc = os.path.join(os.path.dirname(here), "oracle")
    exe = str(tmp_path / "oracle_asan")
    srcs = [os.path.join(orc, f) for f in ("bssn_oracle.c", "bssn_oracle_algebra.c",
                                           "bssn_oracle_algebra_adv.c", "bssn_oracle_constraints.c")]
    subprocess.run(["gcc", "-std=c11", "-O1", "-g", "-fno-omit-frame-pointer", "-ffp-contract=off",
                    "-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-I", orc,
                    os.path.join(here, "oracle_sanitize_main.c"), *srcs, "-o", exe, "-lm"], check=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="print_stacktrace=1")
    out = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "checksum" in out.stdout
