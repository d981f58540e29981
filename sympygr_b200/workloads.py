"""Synthetic BSSN inputs for the parity tests and the benchmark.

Arrays follow the reference's zipped layout: one array per variable (VAR order of
bssn/include/grDef.h:31), each block at an element offset with
IDX(i,j,k) = i + nx*(j + ny*k) (bssn/include/derivs.h:8) and a 3-point ghost layer.

Workloads (seeded, no external data):

* ``flat_sines``     one 38^3 block, h=0.1: flat space (gt=delta, chi=alpha=1, the
                     rest 0) plus, per variable, 4 sine modes with amplitudes
                     U(-1e-3, 1e-3), phases U(0, 2pi) and wavevector components
                     U(1, 4)*2pi/L with L=(n-1)h; ``numpy.random.default_rng(seed*1000+v)``
                     for variable v.  The block is centred on the origin.
* ``brill_lindquist`` one 134^3 block whose 128^3 interior spans [-8, 8]^3; a single
                     puncture of mass 1 at the origin: chi=(1+m/(2r))^-4 with
                     r=sqrt(|x|^2+1e-4), alpha=chi^(1/2), gt=delta, the rest 0;
                     all six faces flagged (bflag 0x3F).
* ``two_puncture_batch`` octree-like batch: padded sizes 13/21/37/69/135 with
                     counts 1800/750/300/120/30 (60/25/10/4/1 %); every block spans
                     the same physical interior width W=1, so h=W/(n-7); block
                     lower interior corners are uniform in [-6, 6-W]^3; the field is
                     a two-puncture Brill-Lindquist data set (m=0.5 at x=+-4,
                     softened as above, alpha=chi^(1/2), gt=delta, the rest 0);
                     10 % of the blocks get a random non-zero face mask.  Block
                     starts are aligned to 32 elements.
* ``tiled_domain_blocks`` blocks of one padded size tiling a cube domain around the
                     same two punctures, the domain's outer faces flagged (Sommerfeld)
                     and the faces between blocks not: the layout of an evolution whose
                     only physical boundary is the outer one.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

NUM_VARS = 24
VAR_NAMES = [
    "alpha", "chi", "K", "Gt0", "Gt1", "Gt2", "beta0", "beta1", "beta2",
    "B0", "B1", "B2", "gt0", "gt1", "gt2", "gt3", "gt4", "gt5",
    "At0", "At1", "At2", "At3", "At4", "At5",
]
U_ALPHA, U_CHI = 0, 1
U_SYMGT0, U_SYMGT3, U_SYMGT5 = 12, 15, 17
FLAT = {U_ALPHA: 1.0, U_CHI: 1.0, U_SYMGT0: 1.0, U_SYMGT3: 1.0, U_SYMGT5: 1.0}

BATCH_SIZES = (13, 21, 37, 69, 135)
BATCH_COUNTS = (1800, 750, 300, 120, 30)


@dataclasses.dataclass
class Block:
    offset: int
    sz: tuple
    bflag: int
    pmin: tuple
    pmax: tuple

    @property
    def npad(self) -> int:
        return self.sz[0] * self.sz[1] * self.sz[2]

    @property
    def ninterior(self) -> int:
        return (self.sz[0] - 6) * (self.sz[1] - 6) * (self.sz[2] - 6)

    @property
    def h(self):
        return tuple((self.pmax[a] - self.pmin[a]) / (self.sz[a] - 1) for a in range(3))


def coords(blk: Block):
    """x, y, z of every padded point, arrays of shape (nz, ny, nx) (x fastest)."""
    h = blk.h
    ax = [blk.pmin[a] + np.arange(blk.sz[a], dtype=np.float64) * h[a] for a in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return x, y, z


def flat_sines(n: int = 38, h: float = 0.1, seed: int = 0):
    """Single block: returns (u [24, n^3] float64, Block)."""
    L = (n - 1) * h
    p0 = -0.5 * L
    blk = Block(0, (n, n, n), 0, (p0,) * 3, (p0 + L,) * 3)
    x, y, z = coords(blk)
    u = np.zeros((NUM_VARS, n * n * n))
    for v in range(NUM_VARS):
        rng = np.random.default_rng(seed * 1000 + v)
        amp = rng.uniform(-1e-3, 1e-3, 4)
        phase = rng.uniform(0.0, 2 * math.pi, 4)
        kvec = rng.uniform(1.0, 4.0, (4, 3)) * (2 * math.pi / L)
        f = np.full(x.shape, FLAT.get(v, 0.0))
        for m in range(4):
            f += amp[m] * np.sin(kvec[m, 0] * x + kvec[m, 1] * y + kvec[m, 2] * z + phase[m])
        u[v] = f.ravel()
    return u, blk


def _bl_fields(u, sl, x, y, z, punctures):
    psi = np.ones_like(x)
    for (px, py, pz, m) in punctures:
        r = np.sqrt((x - px) ** 2 + (y - py) ** 2 + (z - pz) ** 2 + 1e-4)
        psi += m / (2.0 * r)
    chi = psi ** -4
    u[U_CHI, sl] = chi.ravel()
    u[U_ALPHA, sl] = np.sqrt(chi).ravel()
    u[U_SYMGT0, sl] = 1.0
    u[U_SYMGT3, sl] = 1.0
    u[U_SYMGT5, sl] = 1.0


def brill_lindquist(n: int = 134, half_width: float = 8.0, mass: float = 1.0):
    """Single block, all faces flagged: returns (u [24, n^3], Block)."""
    h = 2.0 * half_width / (n - 7)
    p0 = -half_width - 3 * h
    p1 = half_width + 3 * h
    blk = Block(0, (n, n, n), 0x3F, (p0,) * 3, (p1,) * 3)
    x, y, z = coords(blk)
    u = np.zeros((NUM_VARS, n * n * n))
    _bl_fields(u, slice(0, n ** 3), x, y, z, [(0.0, 0.0, 0.0, mass)])
    return u, blk


def batch_blocks(sizes=BATCH_SIZES, counts=BATCH_COUNTS, seed: int = 0, width: float = 1.0,
                 box: float = 6.0, boundary_fraction: float = 0.1, align: int = 32):
    """Block list of the octree-like batch (see module docstring)."""
    rng = np.random.default_rng(seed)
    blocks = []
    off = 0
    for n, c in zip(sizes, counts):
        h = width / (n - 7)
        for _ in range(c):
            lo = rng.uniform(-box, box - width, 3)
            flag = 0
            if rng.uniform() < boundary_fraction:
                flag = int(rng.integers(1, 64))
            pmin = tuple(float(lo[a] - 3 * h) for a in range(3))
            pmax = tuple(float(lo[a] + width + 3 * h) for a in range(3))
            blocks.append(Block(off, (n, n, n), flag, pmin, pmax))
            off += ((n ** 3 + align - 1) // align) * align
    return blocks, off


def two_puncture_batch(sizes=BATCH_SIZES, counts=BATCH_COUNTS, seed: int = 0):
    """Host arrays for the batch: returns (u [24, total] float64, blocks)."""
    blocks, total = batch_blocks(sizes, counts, seed)
    u = np.zeros((NUM_VARS, total))
    punct = [(-4.0, 0.0, 0.0, 0.5), (4.0, 0.0, 0.0, 0.5)]
    for b in blocks:
        x, y, z = coords(b)
        _bl_fields(u, slice(b.offset, b.offset + b.npad), x, y, z, punct)
    return u, blocks


def tiled_domain_blocks(ntile: int = 4, n: int = 37, half_width: float = 8.0, align: int = 32):
    """Blocks of padded size n^3 tiling the cube [-half_width, half_width]^3 with
    ntile^3 blocks: the interiors ((n-6)^3 points each) abut with one spacing h between
    neighbouring interior points, and each block's bflag marks exactly its faces on the
    domain boundary (bits x-, x+, y-, y+, z-, z+ as in the reference's def.h), so the
    Sommerfeld values apply on the outer boundary only.  Returns (blocks, total)."""
    interior = n - 6
    width = 2.0 * half_width / ntile
    h = width / interior
    blocks, off = [], 0
    for bz in range(ntile):
        for by in range(ntile):
            for bx in range(ntile):
                lo = [-half_width + c * width for c in (bx, by, bz)]
                flag = 0
                for a, c in enumerate((bx, by, bz)):
                    if c == 0:
                        flag |= 1 << (2 * a)
                    if c == ntile - 1:
                        flag |= 1 << (2 * a + 1)
                pmin = tuple(lo[a] - 3 * h for a in range(3))
                pmax = tuple(pmin[a] + (n - 1) * h for a in range(3))
                blocks.append(Block(off, (n, n, n), flag, pmin, pmax))
                off += ((n ** 3 + align - 1) // align) * align
    return blocks, off


def two_puncture_fields_torch(blocks, total: int, device="cuda"):
    """The two-puncture Brill-Lindquist fields (m = 0.5 at x = +-4, softened, alpha =
    chi^(1/2), gt = delta, the rest 0) at every padded point of the given blocks,
    built with torch on `device`: a [24, total] tensor."""
    import torch

    u = torch.zeros((NUM_VARS, total), dtype=torch.float64, device=device)
    for v in (U_SYMGT0, U_SYMGT3, U_SYMGT5):
        u[v].fill_(1.0)  # gaps between blocks hold flat values too; never read
    punct = [(-4.0, 0.0, 0.0, 0.5), (4.0, 0.0, 0.0, 0.5)]
    by_size = {}
    for b in blocks:
        by_size.setdefault(b.sz[0], []).append(b)
    for n, bl in by_size.items():
        ar = torch.arange(n, dtype=torch.float64, device=device)
        h = torch.tensor([b.h[0] for b in bl], dtype=torch.float64, device=device)
        pm = torch.tensor([b.pmin for b in bl], dtype=torch.float64, device=device)
        # (nb, n) coordinate lines per axis
        xs = pm[:, 0:1] + ar[None, :] * h[:, None]
        ys = pm[:, 1:2] + ar[None, :] * h[:, None]
        zs = pm[:, 2:3] + ar[None, :] * h[:, None]
        step = max(1, (1 << 26) // (n ** 3))
        for s in range(0, len(bl), step):
            e = min(len(bl), s + step)
            X = xs[s:e, None, None, :]
            Y = ys[s:e, None, :, None]
            Z = zs[s:e, :, None, None]
            psi = torch.ones((e - s, n, n, n), dtype=torch.float64, device=device)
            for (px, py, pz, m) in punct:
                r = torch.sqrt((X - px) ** 2 + (Y - py) ** 2 + (Z - pz) ** 2 + 1e-4)
                psi += m / (2.0 * r)
            chi = psi ** -4
            alpha = torch.sqrt(chi)
            idx = torch.tensor([b.offset for b in bl[s:e]], dtype=torch.int64, device=device)
            flat = (idx[:, None] + torch.arange(n ** 3, device=device)[None, :]).reshape(-1)
            u[U_CHI].index_copy_(0, flat, chi.reshape(-1))
            u[U_ALPHA].index_copy_(0, flat, alpha.reshape(-1))
    return u


def two_puncture_batch_torch(sizes=BATCH_SIZES, counts=BATCH_COUNTS, seed: int = 0,
                             device="cuda"):
    """Same data as ``two_puncture_batch`` built with torch on `device` (fast for
    the full 1.4e8-point batch).  Returns (u tensor [24, total], blocks)."""
    blocks, total = batch_blocks(sizes, counts, seed)
    return two_puncture_fields_torch(blocks, total, device), blocks


def interior_mask(blk: Block):
    """Boolean (nz, ny, nx) mask of the interior [3, n-3)^3."""
    m = np.zeros((blk.sz[2], blk.sz[1], blk.sz[0]), dtype=bool)
    m[3:-3, 3:-3, 3:-3] = True
    return m
