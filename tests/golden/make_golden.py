"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's own CPU bssnrhs (compiled from the reference sources into
oracle/_ref by oracle/Makefile, parity flavour: -O2 -ffp-contract=off) on
seeded inputs and stores its outputs:

* fake_<n>_b<flag>.npz   whole interior RHS of one block filled with the
                         reference's fake_initial_data (bssn/src/grUtils.cpp:15-58)
* sines_38.npz           the 38^3 flat-space + sine-mode block (h=0.1, sigma=0.4):
                         per-variable checksums plus 2048 sampled interior points
* bl_134.npz             the 134^3 Brill-Lindquist block (all faces flagged,
                         sigma=0.4): checksums plus 2048 sampled interior points
* con_fake_<n>_b<flag>.npz  Hamiltonian and momentum constraints (rows ham, mom0,
                         mom1, mom2) at the interior of a fake_initial_data block,
                         from the reference's physical_constraints
                         (bssn/CodeGen/physcon.cpp:12)
* con_bl_70.npz          the same on a 70^3 Brill-Lindquist block: checksums plus
                         2048 sampled interior points
* adv42.npz              the reference's 4th-order upwind advective derivatives
                         deriv42adv_{x,y,z} (bssn/src/derivs.cpp:495-900) of a seeded
                         random 13x15x14 field with a seeded random shift (every 7th
                         value exactly 0), without and with all faces flagged

Each file also records the generator parameters and a SHA-256 of the input
arrays, so a test can verify it regenerated the same inputs.

    python tests/golden/make_golden.py      # needs the reference build (make -C oracle ref)
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import pyoracle as po  # noqa: E402
from sympygr_b200 import workloads as wl  # noqa: E402

FAKE_CASES = [  # (n, pmin, h, bflag)
    (13, (-0.31, -0.22, -0.13), 0.05, 0x00),
    (13, (-0.31, -0.22, -0.13), 0.05, 0x3F),
    (13, (0.4, -0.9, 0.2), 0.07, 0x05),
    (17, (-0.5, 0.1, -0.2), 0.04, 0x2A),
]
SIGMA_FAKE = 0.1
SIGMA_CFG = 0.4
NSAMPLE = 2048


def sha(u: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(u, dtype=np.float64).tobytes()).hexdigest()


def checksums(rint: np.ndarray) -> np.ndarray:
    """Per variable: sum, sum of squares, max |.| over the interior."""
    return np.stack([rint.sum(axis=1), (rint ** 2).sum(axis=1), np.abs(rint).max(axis=1)], axis=1)


def sample_index(npts: int, seed: int) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(npts, NSAMPLE, replace=False))


ADV_H = 0.07


def adv_inputs():
    """Seeded field and shift for the upwind-derivative fixture."""
    sz = (13, 15, 14)
    rng = np.random.default_rng(11)
    n = sz[0] * sz[1] * sz[2]
    f = rng.standard_normal(n)
    beta = rng.standard_normal(n)
    beta[::7] = 0.0
    return f, beta, sz


def main():
    if not po.have_reference("parity"):
        raise SystemExit("reference build missing: make -C oracle ref")
    for n, pmin, h, bflag in FAKE_CASES:
        u, blk = po.fake_block(n, pmin, h, bflag)
        prm = po.params(ko_sigma=SIGMA_FAKE)
        r = po.ref_rhs(u, blk, prm)
        np.savez_compressed(os.path.join(HERE, f"fake_{n}_b{bflag:02x}.npz"),
                            n=n, pmin=np.array(pmin), h=h, bflag=bflag, sigma=SIGMA_FAKE,
                            input_sha=sha(u), rhs_interior=po.interior(r, blk))
        print("fake", n, hex(bflag))
    prm = po.params(ko_sigma=SIGMA_CFG)
    for name, (u, blk), seed in [("sines_38", wl.flat_sines(38, 0.1, 0), 1),
                                 ("bl_134", wl.brill_lindquist(134, 8.0, 1.0), 2)]:
        r = po.ref_rhs(u, blk, prm)
        ri = po.interior(r, blk)
        idx = sample_index(ri.shape[1], seed)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), sigma=SIGMA_CFG, bflag=blk.bflag,
                            input_sha=sha(u), checksums=checksums(ri), sample_index=idx,
                            sample_rhs=ri[:, idx])
        print(name, blk.sz, hex(blk.bflag))
    for n, pmin, h, bflag in (FAKE_CASES[0], FAKE_CASES[3]):
        u, blk = po.fake_block(n, pmin, h, bflag)
        c = po.interior(po.ref_constraints(u, blk), blk)[:4]
        np.savez_compressed(os.path.join(HERE, f"con_fake_{n}_b{bflag:02x}.npz"),
                            n=n, pmin=np.array(pmin), h=h, bflag=bflag, input_sha=sha(u),
                            con_interior=c)
        print("constraints fake", n, hex(bflag))
    u, blk = wl.brill_lindquist(70, 8.0, 1.0)
    c = po.interior(po.ref_constraints(u, blk), blk)[:4]
    idx = sample_index(c.shape[1], 3)
    np.savez_compressed(os.path.join(HERE, "con_bl_70.npz"), bflag=blk.bflag, input_sha=sha(u),
                        checksums=checksums(c), sample_index=idx, sample_con=c[:, idx])
    print("constraints bl_70", blk.sz)
    f, beta, sz = adv_inputs()
    outs = {f"d{axis}_b{bflag:02x}": po.ref_deriv42adv(axis, f, ADV_H, sz, beta, bflag)
            for axis in range(3) for bflag in (0x00, 0x3F)}
    np.savez_compressed(os.path.join(HERE, "adv42.npz"), h=ADV_H, sz=np.array(sz),
                        input_sha=sha(np.concatenate([f, beta])), **outs)
    print("adv42", sz)


if __name__ == "__main__":
    main()
