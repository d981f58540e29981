"""CPU: the tiled-domain layout of the evolution driver -- abutting interiors, face
flags on the domain boundary only."""
from sympygr_b200 import workloads as wl


def test_tiled_domain_geometry():
    blocks, total = wl.tiled_domain_blocks(3, 21, 6.0)
    assert len(blocks) == 27 and total >= 27 * 21 ** 3
    h = blocks[0].h[0]
    for b in blocks:
        assert all(abs(x - h) < 1e-12 for x in b.h)
    # x neighbours: the first interior point of the next block is one spacing on
    assert abs((blocks[0].pmin[0] + 17 * h + h) - (blocks[1].pmin[0] + 3 * h)) < 1e-12
    # the interiors span the domain
    assert abs(blocks[0].pmin[0] + 3 * h + 6.0) < 1e-12
    last = blocks[-1]
    assert abs(last.pmin[0] + (21 - 4) * h - (6.0 - h)) < 1e-12
    # flags: the centre block none, a corner block three faces, each face bit once per side
    assert blocks[13].bflag == 0
    assert blocks[0].bflag == 0x15 and blocks[26].bflag == 0x2A
    for bit in range(6):
        assert sum(1 for b in blocks if b.bflag >> bit & 1) == 9
