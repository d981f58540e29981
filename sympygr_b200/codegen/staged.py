"""Staged capture of the BSSN right-hand side from the reference's SymPy layer.

``symbolic_source.capture_bssn_rhs`` returns the 24 outputs fully expanded in
the state variables and their derivatives; one global CSE over them leaves the
Ricci tensor spread over ~450 temporaries that all six At_rhs components share,
so a device function needs ~540 live values.  Here the same construction
(GR/bssn.py:57-105 on top of GR/dendro.py) is run with the geometric
intermediates replaced by symbols, in the order the mathematics builds them:

    igt   inverse conformal metric        dendro.get_inverse_metric   (dendro.py:364)
    C1    first-kind Christoffels of gt   dendro.get_first_christoffel (:380)
    C2    second-kind Christoffels        dendro.get_second_christoffel (:403)
    CalGt contracted connection           dendro.compute_ricci        (:488)
    C3    Christoffels of gt/chi          dendro.get_complete_christoffel (:422)
    R     Ricci tensor                    dendro.compute_ricci        (:451-521)
    out   the 24 right-hand sides         GR/bssn.py:67-98

Each stage's definitions are expressions in the inputs and the earlier stages'
symbols, so every stage can be CSE'd on its own and its temporaries die before
the next stage starts; only the ~70 stage values cross stage boundaries.  The
physics is unchanged: substituting the stage definitions back reproduces the
reference's expressions, and the generated code is checked numerically against
the reference's bssnrhs.
"""
from __future__ import annotations

import contextlib
import io
import os
import sys

import sympy as sp
from sympy.tensor.array import MutableDenseNDimArray

from .symbolic_source import _MAT_IDX, _MAT_SUF, _rename

PAIRS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]


def _sym3(name):
    """Symmetric 3x3 Matrix of symbols name00..name22."""
    s = {p: sp.Symbol(f"{name}{p[0]}{p[1]}") for p in PAIRS}
    return sp.Matrix(3, 3, lambda i, j: s[(min(i, j), max(i, j))])


def _chris(name):
    """3x3x3 array X[k, i, j] of symbols, symmetric in (i, j)."""
    arr = MutableDenseNDimArray(range(27), (3, 3, 3))
    for k in range(3):
        for i in range(3):
            for j in range(3):
                a, b = min(i, j), max(i, j)
                arr[k, i, j] = sp.Symbol(f"{name}_{k}_{a}{b}")
    return arr


def capture_constraints_staged(reference_root: str):
    """Hamiltonian and momentum constraints of GR/constraints.py:166-177 with the
    same stage symbols (igt, C1, C2, CalGt, R; the stage definitions are those of
    ``capture_staged``).  Returns [(stage_name, defs), ..., ("out", [(name, expr)])]
    with outputs ham, mom0, mom1, mom2.  Must run after ``capture_staged`` in the
    same process (it reuses the symbolic dendro state that function leaves)."""
    import dendro  # GR/dendro.py, already configured with the stage symbols

    Rs = _sym3("R")
    CalGts = [sp.Symbol(f"CalGt{i}") for i in range(3)]
    saved = dendro.compute_ricci
    dendro.compute_ricci = lambda Gt_, chi_: [Rs, None, None, CalGts]
    try:
        import importlib

        if "constraints" in sys.modules:
            con = importlib.reload(sys.modules["constraints"])
        else:
            import constraints as con  # GR/constraints.py
    finally:
        dendro.compute_ricci = saved
    outs = [("ham", con.ham)] + [(f"mom{i}", con.mom[i]) for i in range(3)]
    return [("out", [(n, _rename(sp.sympify(e))) for n, e in outs])]


def capture_staged(reference_root: str):
    """Returns a list of stages [(stage_name, [(symbol, expr), ...]), ...]; the last
    stage holds the 24 outputs as (output_name, expr).  Expressions use the plain
    identifiers of ``symbolic_source._rename``."""
    gr = os.path.join(reference_root, "GR")
    if gr not in sys.path:
        sys.path.insert(0, gr)
    import dendro  # GR/dendro.py
    import bssn as bssn_sym  # GR/bssn.py (builds the metric and its inverse at import)

    IGT = _sym3("igt")
    C1s, C2s, C3s = _chris("C1"), _chris("C2"), _chris("C3")
    CalGts = [sp.Symbol(f"CalGt{i}") for i in range(3)]
    Rs = _sym3("R")
    chi = bssn_sym.chi
    Gt = bssn_sym.Gt

    stages = []
    # inverse metric: the reference's own expression (bssn.py:47 -> dendro.py:375)
    igt_full = dendro.get_inverse_metric()
    stages.append(("igt", [(IGT[i, j], igt_full[i, j]) for i, j in PAIRS]))
    dendro.inv_metric = IGT

    dendro.C1 = dendro.undef
    c1 = dendro.get_first_christoffel()
    stages.append(("C1", [(C1s[k, i, j], c1[k, i, j]) for k in range(3) for i, j in PAIRS]))
    dendro.C1 = C1s

    dendro.C2 = dendro.undef
    c2 = dendro.get_second_christoffel()
    stages.append(("C2", [(C2s[k, i, j], c2[k, i, j]) for k in range(3) for i, j in PAIRS]))
    dendro.C2 = C2s

    # Ricci tensor and CalGt with the symbolic Christoffels (dendro.py:451-521)
    R_full, _, _, calgt = dendro.compute_ricci(Gt, chi)
    stages.append(("CalGt", [(CalGts[i], calgt[i]) for i in range(3)]))

    dendro.C3 = dendro.undef
    c3 = dendro.get_complete_christoffel(chi)
    stages.append(("C3", [(C3s[k, i, j], c3[k, i, j]) for k in range(3) for i, j in PAIRS]))
    dendro.C3 = C3s

    stages.append(("R", [(Rs[i, j], R_full[i, j]) for i, j in PAIRS]))

    # the right-hand side, with compute_ricci answering with the stage symbols
    captured = {}

    def recorder(ex, vnames, idx):
        captured["ex"], captured["vnames"] = ex, vnames

    saved_gen, saved_ricci, saved_igt = dendro.generate_cpu, dendro.compute_ricci, bssn_sym.igt
    dendro.generate_cpu = recorder
    dendro.compute_ricci = lambda Gt_, chi_: [Rs, None, None, CalGts]
    bssn_sym.igt = IGT
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            bssn_sym.bssn_puncture_gauge(bssn_sym.eta, False)
    finally:
        dendro.generate_cpu, dendro.compute_ricci, bssn_sym.igt = saved_gen, saved_ricci, saved_igt

    outs = []
    for e, vname in zip(captured["ex"], captured["vnames"]):
        if isinstance(e, list):
            outs += [(f"{vname}{j}", ev) for j, ev in enumerate(e)]
        elif isinstance(e, sp.MatrixBase):
            outs += [(f"{vname}{_MAT_SUF[j]}", e[k]) for j, k in enumerate(_MAT_IDX)]
        else:
            outs.append((vname, e))
    stages = [(name, [(s, _rename(sp.sympify(e))) for s, e in defs]) for name, defs in stages]
    stages.append(("out", [(n, _rename(sp.sympify(e))) for n, e in outs]))
    return stages
