"""sympygr_b200: B200-native BSSN right-hand side for Dendro octree blocks.

The product is the CUDA library ``lib/libb200bssn.so`` (C ABI in
include/b200bssn.h).  This package holds its build script, the code generator
that prints the per-point algebra, synthetic workloads, and a thin ctypes mirror
of the reference's entry point:

    import sympygr_b200 as sg
    ctx = sg.Context(0)
    sg.bssnrhs(ctx, rhs, u, offset, ptmin, ptmax, sz, bflag, params)

which follows ``bssnrhs(uzipVarsRHS, uZipVars, offset, ptmin, ptmax, sz, bflag)``
(bssn/include/rhs.h:33-36).
"""
from .capi import (FP64, GHOSTS_PRESERVE, GHOSTS_ZERO, MIXED, RK4, B200BssnError, Context, Params,
                   Plan, load)
from .workloads import Block

__all__ = ["Context", "Plan", "RK4", "Params", "Block", "B200BssnError", "FP64", "MIXED",
           "GHOSTS_PRESERVE", "GHOSTS_ZERO", "bssnrhs", "load"]


def bssnrhs(ctx, rhs, u, offset, ptmin, ptmax, sz, bflag, params=None):
    """Reference-shaped entry point on host arrays; see ``Context.bssnrhs``."""
    if params is None:
        params = Params.make()
    ctx.bssnrhs(rhs, u, offset, ptmin, ptmax, sz, bflag, params)
