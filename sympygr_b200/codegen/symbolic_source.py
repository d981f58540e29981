"""Capture the BSSN right-hand-side expressions from the reference's symbolic layer.

The reference builds its per-point algebra in SymPy (GR/bssn.py:57-105,
``bssn_puncture_gauge``) on top of the helper module GR/dendro.py, then hands the
expression list to ``dendro.generate_cpu`` (GR/dendro.py:567-623), which runs CSE
and prints C++.  This module drives the same SymPy construction but intercepts the
hand-off: ``generate_cpu`` is replaced by a recorder, so the expressions come out
as SymPy objects that our own printers (C for the oracle, CUDA for the kernels) can
consume.  The expression construction itself is the reference's own code, so the
physics (gauge, damping, Lie derivatives, Ricci tensor) is exactly what the
reference's committed bssneqs_eta_const_standard_gauge.cpp was generated from.

Only used at code-generation time, where the reference tree is available.
"""
from __future__ import annotations

import contextlib
import io
import os
import re
import sys
import types

import sympy as sp

# Output naming follows GR/dendro.py:579-596: lists get a numeric suffix, symmetric
# 3x3 matrices the entries [0,1,2,4,5,8] with suffixes 00,01,02,11,12,22.
_MAT_IDX = [0, 1, 2, 4, 5, 8]
_MAT_SUF = ["00", "01", "02", "11", "12", "22"]

# VAR enum of the reference (bssn/include/grDef.h:31) and the array names used by
# bssnrhs for each variable (bssn/src/rhs.cpp:88-135).
VAR_NAMES = [
    "alpha", "chi", "K", "Gt0", "Gt1", "Gt2", "beta0", "beta1", "beta2",
    "B0", "B1", "B2", "gt0", "gt1", "gt2", "gt3", "gt4", "gt5",
    "At0", "At1", "At2", "At3", "At4", "At5",
]
RHS_NAMES = [
    "a_rhs", "chi_rhs", "K_rhs", "Gt_rhs0", "Gt_rhs1", "Gt_rhs2",
    "b_rhs0", "b_rhs1", "b_rhs2", "B_rhs0", "B_rhs1", "B_rhs2",
    "gt_rhs00", "gt_rhs01", "gt_rhs02", "gt_rhs11", "gt_rhs12", "gt_rhs22",
    "At_rhs00", "At_rhs01", "At_rhs02", "At_rhs11", "At_rhs12", "At_rhs22",
]
# Variables that get second derivatives (bssn/scripts/gen_bssnrhs_code:31-32).
DD_VARS = ["gt0", "gt1", "gt2", "gt3", "gt4", "gt5", "chi", "alpha", "beta0", "beta1", "beta2"]
DD_PAIRS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]


def derivative_slots():
    """Slot table of the derivative scratch, in storage order.

    72 first derivatives (24 vars x 3 directions, VAR order), then 66 second
    derivatives (11 vars x 6 index pairs), then 24 Kreiss-Oliger sums.  The first
    138 entries are the arrays that bssnrhs materialises
    (bssn/scripts/bssnrhs_derivs.h); the last 24 hold ko_x+ko_y+ko_z of each
    variable (bssn/src/rhs.cpp:332-369 sums the three KO arrays).
    """
    slots = []
    for v in VAR_NAMES:
        for d in range(3):
            slots.append(f"grad_{d}_{v}")
    for v in DD_VARS:
        for a, b in DD_PAIRS:
            slots.append(f"grad2_{a}_{b}_{v}")
    for v in VAR_NAMES:
        slots.append(f"kosum_{v}")
    return slots


# The advective derivatives agrad_* (bssn/scripts/bssnrhs_derivs_adv.h) are the same
# arrays as grad_* in the reference's default 6th-order build, where deriv64adv_* is
# deriv64_* (bssn/src/derivs.cpp:2841-2881).  With ADVECTIVE set, _rename keeps them as
# their own symbols agrad_<d>_<var>, for the opt-in upwind mode.
ADVECTIVE = False


def advective_slots():
    """The 72 advective-derivative slots of the upwind mode, VAR order, x/y/z."""
    return [f"agrad_{d}_{v}" for v in VAR_NAMES for d in range(3)]


def _install_import_stubs():
    """dendrosym imports tomlkit and matplotlib, neither needed for printing."""
    if "tomlkit" not in sys.modules:
        tk = types.ModuleType("tomlkit")
        tk.table = dict
        tk.Table = dict
        tk.document = dict
        tk.items = types.SimpleNamespace(Table=dict)
        sys.modules["tomlkit"] = tk
        sys.modules["tomlkit.items"] = tk.items
    if "matplotlib" not in sys.modules:
        mpl = types.ModuleType("matplotlib")
        plt = types.ModuleType("matplotlib.pyplot")
        mpl.pyplot = plt
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = plt
    if "git" not in sys.modules:
        sys.modules["git"] = types.ModuleType("git")


def load_dendro_c_printer(reference_root: str):
    """Return the reference's ``DendroCPrinter`` class (dendrosym/code_printer.py:9)."""
    _install_import_stubs()
    if reference_root not in sys.path:
        sys.path.insert(0, reference_root)
    from dendrosym.code_printer import DendroCPrinter  # noqa: E402

    return DendroCPrinter


def capture_bssn_rhs(reference_root: str):
    """Run GR/bssn.py's ``bssn_puncture_gauge(eta, isStaged=False)`` and capture
    the 24 output expressions it would print.

    Returns ``(names, exprs)`` with ``names`` in the reference's output naming
    (``a_rhs``, ``b_rhs0`` ... ``B_rhs2``) and ``exprs`` as SymPy expressions in
    which every array access ``f[pp]`` is a plain Symbol ``f`` and every stencil
    call is a Symbol named after the derivative array that holds it
    (``grad_0_alpha``, ``grad2_0_1_gt0``; ``agrad_*`` is mapped to ``grad_*`` as in
    the default build, bssn/scripts/bssnrhs_memalloc_adv.h).
    """
    gr = os.path.join(reference_root, "GR")
    if gr not in sys.path:
        sys.path.insert(0, gr)
    import dendro  # GR/dendro.py
    import bssn as bssn_sym  # GR/bssn.py

    captured = {}

    def recorder(ex, vnames, idx):
        captured["ex"] = ex
        captured["vnames"] = vnames
        captured["idx"] = idx

    saved = dendro.generate_cpu
    dendro.generate_cpu = recorder
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            bssn_sym.bssn_puncture_gauge(bssn_sym.eta, False)
    finally:
        dendro.generate_cpu = saved

    names, exprs = [], []
    for e, vname in zip(captured["ex"], captured["vnames"]):
        if isinstance(e, list):
            for j, ev in enumerate(e):
                names.append(f"{vname}{j}")
                exprs.append(ev)
        elif isinstance(e, sp.MatrixBase):
            for j, k in enumerate(_MAT_IDX):
                names.append(f"{vname}{_MAT_SUF[j]}")
                exprs.append(e[k])
        else:
            names.append(vname)
            exprs.append(e)
    exprs = [_rename(e) for e in exprs]
    return names, exprs


_ARR = re.compile(r"^(\w+)\[pp\]$")
_PAR = re.compile(r"^(\w+)\[(\d)\]$")


def _rename(expr):
    """Map reference symbols to plain identifiers (see ``capture_bssn_rhs``)."""
    rep = {}
    for s in expr.free_symbols:
        m = _ARR.match(s.name)
        if m:
            rep[s] = sp.Symbol(m.group(1))
            continue
        m = _PAR.match(s.name)
        if m:  # lambda[0] -> lambda0, lambda_f[1] -> lambda_f1
            rep[s] = sp.Symbol(m.group(1) + m.group(2))
    expr = expr.xreplace(rep)
    frep = {}
    for f in expr.atoms(sp.Function):
        fname = type(f).__name__
        if fname in ("grad", "agrad", "kograd"):
            d, var = f.args
            prefix = "agrad" if (fname == "agrad" and ADVECTIVE) else "grad"
            frep[f] = sp.Symbol(f"{prefix}_{int(d)}_{var.name}")
        elif fname == "grad2":
            a, b, var = f.args
            a, b = sorted((int(a), int(b)))
            frep[f] = sp.Symbol(f"grad2_{a}_{b}_{var.name}")
    return expr.xreplace(frep)


def capture_constraints(reference_root: str):
    """The Hamiltonian and momentum constraints of GR/constraints.py:166-177
    (``ham``, ``mom``), fully expanded in the state and its derivatives.  Must run
    before ``staged.capture_staged`` in a process (that function replaces dendro's
    geometric quantities by symbols)."""
    gr = os.path.join(reference_root, "GR")
    if gr not in sys.path:
        sys.path.insert(0, gr)
    with contextlib.redirect_stdout(io.StringIO()):
        import constraints as con  # GR/constraints.py (builds the expressions at import)
    names = ["ham", "mom0", "mom1", "mom2"]
    exprs = [con.ham] + [con.mom[i] for i in range(3)]
    return names, [_rename(sp.sympify(e)) for e in exprs]
