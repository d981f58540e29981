"""Generate the per-point BSSN algebra for the CUDA kernels and the C oracle.

Pipeline (run where the reference tree is available; outputs are committed):

1. ``symbolic_source.capture_bssn_rhs`` runs the reference's own SymPy
   construction (GR/bssn.py:57-105, standard gauge, constant eta damping, the
   configuration bssn/src/rhs.cpp:224-243 compiles by default) and returns the 24
   right-hand-side expressions.
2. ``sympy.cse`` with ``optimizations='basic'``, as GR/dendro.py:559-562 does.
3. Statements are ordered so that each input is read just before its first use
   and each output is emitted as soon as its last temporary exists, which keeps
   the live set of the device function small.
4. ``CudaPrinter`` (a ``DendroCPrinter`` subclass, see cuda_printer.py) prints a
   precision-generic device template; ``CPrinter`` prints the oracle's C twin.

Usage::

    python -m sympygr_b200.codegen.gen_bssn_rhs --reference /path/to/SymPyGR
    python -m sympygr_b200.codegen.gen_bssn_rhs --reference /path/to/SymPyGR --advective
"""
from __future__ import annotations

import argparse
import os
import pickle
import time

import sympy as sp

from . import symbolic_source as src
from .cuda_printer import make_printers

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
CUDA_OUT = os.path.join(REPO, "sympygr_b200", "csrc", "generated", "bssn_rhs_algebra.cuh")
C_OUT = os.path.join(REPO, "oracle", "bssn_oracle_algebra.c")
CUDA_CON_OUT = os.path.join(REPO, "sympygr_b200", "csrc", "generated", "bssn_constraints_algebra.cuh")
C_CON_OUT = os.path.join(REPO, "oracle", "bssn_oracle_constraints.c")
CUDA_ADV_OUT = os.path.join(REPO, "sympygr_b200", "csrc", "generated", "bssn_rhs_algebra_adv.cuh")
C_ADV_OUT = os.path.join(REPO, "oracle", "bssn_oracle_algebra_adv.c")
CON_NAMES = ["ham", "mom0", "mom1", "mom2"]
CON_INDEX = {n: i for i, n in enumerate(CON_NAMES)}

PARAM_NAMES = ["lambda0", "lambda1", "lambda2", "lambda3", "lambda_f0", "lambda_f1"]

# rhs output name -> VAR index (bssn/include/grDef.h:31, bssn/src/rhs.cpp:113-136)
OUT_VAR = {n: i for i, n in enumerate(src.RHS_NAMES)}


def schedule(names, repl, reduced):
    """Order CSE statements: temporaries in dependency order (as CSE returns them),
    each output placed right after the temporary that completes it, and each
    input symbol bound immediately before its first reader.

    Returns a list of ("in", sym) / ("tmp", sym, expr) / ("out", name, expr).
    """
    tmp_index = {s: i for i, (s, _) in enumerate(repl)}
    # outputs keyed by the last temporary they need
    ready_after = {}
    for name, e in zip(names, reduced):
        deps = [tmp_index[s] for s in e.free_symbols if s in tmp_index]
        key = max(deps) if deps else -1
        ready_after.setdefault(key, []).append((name, e))
    seen_inputs = set()
    prog = []

    def bind_inputs(expr):
        for s in sorted(expr.free_symbols, key=lambda x: x.name):
            if s in tmp_index or s in seen_inputs:
                continue
            seen_inputs.add(s)
            prog.append(("in", s))

    for name, e in ready_after.get(-1, []):
        bind_inputs(e)
        prog.append(("out", name, e))
    for i, (s, e) in enumerate(repl):
        bind_inputs(e)
        prog.append(("tmp", s, e))
        for name, oe in ready_after.get(i, []):
            bind_inputs(oe)
            prog.append(("out", name, oe))
    return prog


def _input_binding(sym_name, slots, flavor):
    """Source of an input symbol: state value, derivative slot, or parameter."""
    if sym_name in src.VAR_NAMES:
        v = src.VAR_NAMES.index(sym_name)
        return ("in.u(%d)" % v) if flavor == "cuda" else ("u[%d]" % v)
    if sym_name in slots:
        k = slots.index(sym_name)
        return ("in.d(%d)" % k) if flavor == "cuda" else ("d[%d]" % k)
    if sym_name in PARAM_NAMES:
        k = PARAM_NAMES.index(sym_name)
        return ("prm.%s" % sym_name) if flavor == "cuda" else ("par[%d]" % k)
    if sym_name == "eta":
        return "eta"
    raise KeyError(sym_name)


def emit_staged(stages, printer, slots, out_index=None):
    """CUDA body for the staged capture (staged.py): each stage is CSE'd on its own
    and its values are bound to named locals before the next stage starts; the
    last stage's outputs go to the sink (index from `out_index`, default the RHS
    VAR order).  Returns (lines, ops after CSE, temps)."""
    out_index = OUT_VAR if out_index is None else out_index
    lines = []
    seen_inputs = set()
    nops = ntmp = 0
    stage_syms = set()
    for si, (name, defs) in enumerate(stages):
        syms = [d[0] for d in defs]
        exprs = [d[1] for d in defs]
        repl, reduced = sp.cse(exprs, symbols=sp.numbered_symbols(f"s{si}_t"), optimizations="basic")
        ntmp += len(repl)
        lines.append("  // ---- stage %s: %d values, %d temporaries" % (name, len(defs), len(repl)))
        last = name == "out"
        tmp_index = {t: i for i, (t, _) in enumerate(repl)}
        ready_after = {}
        for sym, e in zip(syms, reduced):
            deps = [tmp_index[x] for x in e.free_symbols if x in tmp_index]
            ready_after.setdefault(max(deps) if deps else -1, []).append((sym, e))

        def bind(expr):
            for x in sorted(expr.free_symbols, key=lambda z: z.name):
                if x in tmp_index or x in seen_inputs or x in stage_syms or x.name == "eta":
                    continue
                seen_inputs.add(x)
                lines.append("  const RT %s = %s;" % (x.name, _input_binding(x.name, slots, "cuda")))

        def put(sym, e):
            nonlocal nops
            nops += sp.count_ops(e)
            bind(e)
            if last:
                lines.append("  sink.put(%d, %s);  // %s" % (out_index[sym], printer.doprint(e), sym))
            else:
                lines.append("  const RT %s = %s;" % (sym.name, printer.doprint(e)))
                stage_syms.add(sym)

        for sym, e in ready_after.get(-1, []):
            put(sym, e)
        for i, (t, e) in enumerate(repl):
            nops += sp.count_ops(e)
            bind(e)
            lines.append("  const RT %s = %s;" % (t.name, printer.doprint(e)))
            for sym, oe in ready_after.get(i, []):
                put(sym, oe)
    return lines, nops, ntmp


def emit(prog, printer, flavor, slots, out_index=None):
    out_index = OUT_VAR if out_index is None else out_index
    lines = []
    rt = "RT" if flavor == "cuda" else "double"
    nops = 0
    for item in prog:
        if item[0] == "in":
            s = item[1]
            if s.name == "eta":
                continue
            lines.append("  const %s %s = %s;" % (rt, s.name, _input_binding(s.name, slots, flavor)))
        elif item[0] == "tmp":
            _, s, e = item
            nops += sp.count_ops(e)
            lines.append("  const %s %s = %s;" % (rt, s.name, printer.doprint(e)))
        else:
            _, name, e = item
            nops += sp.count_ops(e)
            v = out_index[name]
            if flavor == "cuda":
                lines.append("  sink.put(%d, %s);  // %s" % (v, printer.doprint(e), name))
            else:
                lines.append("  out[%d] = %s;  /* %s */" % (v, printer.doprint(e), name))
    return lines, nops


CUDA_HEADER = """\
// GENERATED by sympygr_b200/codegen/gen_bssn_rhs.py -- do not edit by hand.
//
// Per-point BSSN right-hand side, standard gauge with constant eta damping: the
// expressions of GR/bssn.py:57-105 (bssn_puncture_gauge), CSE'd with
// sympy.cse(optimizations='basic') and printed by CudaPrinter (a subclass of
// dendrosym/code_printer.py:DendroCPrinter).  It computes what the reference's
// bssn/src/bssneqs_eta_const_standard_gauge.cpp computes (%(orig)s original ops,
// %(nops)d after CSE here, %(ntmp)d temporaries).
//
// Interface:
//   In   : in.u(v)  -> RT   state variable v (VAR order of bssn/include/grDef.h:31)
//          in.d(s)  -> RT   derivative slot s (slot table: 72 first, 66 second)
//   Sink : sink.put(v, RT)  right-hand side of variable v
//   prm  : lambda0..3, lambda_f0..1 (bssn::BSSN_LAMBDA, bssn::BSSN_LAMBDA_F)
//   eta  : the damping factor of B_rhs at this point (bssn/src/rhs.cpp:215-219)
#pragma once

namespace b200bssn {

template <typename RT>
struct AlgebraParams {
  RT lambda0, lambda1, lambda2, lambda3, lambda_f0, lambda_f1;
};

template <typename RT, class In, class Sink>
__device__ __forceinline__ void bssn_rhs_algebra(const In& in, Sink& sink,
                                                 const AlgebraParams<RT>& prm, const RT eta) {
"""

CUDA_HEADER_STAGED = CUDA_HEADER.replace(
    "// expressions of GR/bssn.py:57-105 (bssn_puncture_gauge), CSE'd with\n"
    "// sympy.cse(optimizations='basic') and printed by CudaPrinter (a subclass of\n"
    "// dendrosym/code_printer.py:DendroCPrinter).",
    "// expressions of GR/bssn.py:57-105 (bssn_puncture_gauge), built in stages\n"
    "// (inverse metric, Christoffels, CalGt, Ricci tensor, outputs; see\n"
    "// sympygr_b200/codegen/staged.py), each stage CSE'd on its own with\n"
    "// sympy.cse(optimizations='basic') and printed by CudaPrinter (a subclass of\n"
    "// dendrosym/code_printer.py:DendroCPrinter).")

CUDA_CON_HEADER = """\
// GENERATED by sympygr_b200/codegen/gen_bssn_rhs.py -- do not edit by hand.
//
// Hamiltonian and momentum constraints of GR/constraints.py:166-177
// (ham = chi igt^jk R_jk - A_ij A^ij + 2/3 K^2, mom_i), built in the same stages
// as the right-hand side (inverse metric, Christoffels, CalGt, Ricci tensor; see
// sympygr_b200/codegen/staged.py), each stage CSE'd with
// sympy.cse(optimizations='basic') and printed by CudaPrinter.  %(nops)d ops.
//
// Interface: as bssn_rhs_algebra; sink.put(c, RT) with c = 0 ham, 1..3 mom0..2.
#pragma once

namespace b200bssn {

template <typename RT, class In, class Sink>
__device__ __forceinline__ void bssn_constraints_algebra(const In& in, Sink& sink) {
"""

C_CON_HEADER = """\
/* TEST INFRASTRUCTURE ONLY (oracle).
 * GENERATED by sympygr_b200/codegen/gen_bssn_rhs.py -- do not edit by hand.
 *
 * C restatement of the Hamiltonian and momentum constraints of
 * GR/constraints.py:166-177 (the expressions bssn/CodeGen/physcon.cpp was generated
 * from), expanded in the state and its derivatives, CSE'd with
 * sympy.cse(optimizations='basic') and printed in C99 double arithmetic.
 *
 *   u[24], d[138]  as bssn_oracle_algebra;   out[4]  ham, mom0, mom1, mom2
 */
#include <math.h>
#include "bssn_oracle.h"

void bssn_oracle_constraints(const double *u, const double *d, double *out) {
"""

C_HEADER = """\
/* TEST INFRASTRUCTURE ONLY (oracle).
 * GENERATED by sympygr_b200/codegen/gen_bssn_rhs.py -- do not edit by hand.
 *
 * C restatement of the reference's per-point algebra
 * bssn/src/bssneqs_eta_const_standard_gauge.cpp (included by bssnrhs at
 * bssn/src/rhs.cpp:240): the same SymPy expressions (GR/bssn.py:57-105), CSE'd
 * with sympy.cse(optimizations='basic') as GR/dendro.py:559-562 does, printed in
 * C99 double arithmetic.  %(orig)s original ops, %(nops)d after CSE.
 *
 *   u[24]   state values at the point (VAR order, bssn/include/grDef.h:31)
 *   d[138]  derivatives: grad_{0,1,2}_<var> for the 24 vars, then
 *           grad2_{00,01,02,11,12,22}_<var> for gt0..gt5, chi, alpha, beta0..2
 *   par[6]  lambda[0..3], lambda_f[0..1]
 *   eta     damping factor at the point (bssn/src/rhs.cpp:215-219)
 *   out[24] right-hand sides (VAR order)
 */
#include <math.h>
#include "bssn_oracle.h"

void bssn_oracle_algebra(const double *u, const double *d, const double *par, double eta,
                         double *out) {
"""


CUDA_ADV_HEADER = """\
// GENERATED by sympygr_b200/codegen/gen_bssn_rhs.py --advective -- do not edit by hand.
//
// The per-point BSSN right-hand side of bssn_rhs_algebra.cuh with the advective
// derivatives (the beta^i d_i terms, agrad_* in GR/bssn.py) read from their own slots
// 138..209 (agrad_<d>_<var>, VAR order, x/y/z) instead of the centred first
// derivatives: the opt-in upwind mode, where they come from the 4th-order upwind
// stencils (bssn/src/derivs.cpp:495-900).  Built in the same stages, %(nops)d ops,
// %(ntmp)d temporaries.  Interface as bssn_rhs_algebra.
#pragma once

#include "bssn_rhs_algebra.cuh"

namespace b200bssn {

template <typename RT, class In, class Sink>
__device__ __forceinline__ void bssn_rhs_algebra_adv(const In& in, Sink& sink,
                                                     const AlgebraParams<RT>& prm, const RT eta) {
"""

C_ADV_HEADER = """\
/* TEST INFRASTRUCTURE ONLY (oracle).
 * GENERATED by sympygr_b200/codegen/gen_bssn_rhs.py --advective -- do not edit by hand.
 *
 * bssn_oracle_algebra with the advective derivatives in their own slots:
 *   d[210]  d[0..137] as bssn_oracle_algebra, d[138 + 3*v + k] = agrad_k of VAR v
 * (the beta^i d_i terms of GR/bssn.py, which the reference's default build feeds
 * with the centred first derivatives).  %(nops)d ops after CSE.
 */
#include <math.h>
#include "bssn_oracle.h"

void bssn_oracle_algebra_adv(const double *u, const double *d, const double *par, double eta,
                             double *out) {
"""


def main_advective(args):
    """The upwind-mode algebra (agrad slots separate): CUDA staged + C flat."""
    src.ADVECTIVE = True
    slots = src.derivative_slots()[:138] + src.advective_slots()
    CudaPrinter, CPrinter = make_printers(src.load_dendro_c_printer(args.reference))
    t0 = time.time()
    names, exprs = src.capture_bssn_rhs(args.reference)
    repl, reduced = sp.cse(exprs, symbols=sp.numbered_symbols("t"), optimizations="basic")
    print("advective: captured + cse: %.1fs, %d temporaries" % (time.time() - t0, len(repl)))
    body, nops = emit(schedule(names, repl, reduced), CPrinter(), "c", slots)
    with open(C_ADV_OUT, "w") as f:
        f.write(C_ADV_HEADER % {"nops": nops})
        f.write("\n".join(body))
        f.write("\n}\n")
    from .staged import capture_staged

    stages = capture_staged(args.reference)
    body, nops, ntmp = emit_staged(stages, CudaPrinter(), slots)
    with open(CUDA_ADV_OUT, "w") as f:
        f.write(CUDA_ADV_HEADER % {"nops": nops, "ntmp": ntmp})
        f.write("\n".join(body))
        f.write("\n}\n\n}  // namespace b200bssn\n")
    print("wrote", CUDA_ADV_OUT, "and", C_ADV_OUT)


CUDA_SPLIT_HEADER = """\
// GENERATED by sympygr_b200/codegen/gen_bssn_rhs.py --split -- do not edit by hand.
//
// The per-point BSSN right-hand side of bssn_rhs_algebra.cuh partitioned by output,
// as the reference's staged bssnrhs_sep (bssn/src/rhs.cpp:392-825) partitions its
// loops: part 0 writes the six At_rhs (the only outputs that need the Ricci
// tensor), part 1 the other 18.  Each part carries only the stages its outputs use
// (the staged capture of sympygr_b200/codegen/staged.py, pruned backwards from the
// outputs) and is CSE'd on its own, so the live set of either is a fraction of the
// whole: a register-pressure split for the FP64 algebra.  Part 0: %(nops0)d ops,
// %(ntmp0)d temporaries; part 1: %(nops1)d ops, %(ntmp1)d temporaries.
// Interface as bssn_rhs_algebra; part 0 needs no parameters and no eta.
#pragma once

#include "bssn_rhs_algebra.cuh"

namespace b200bssn {

template <int PART>
struct RhsAlgebraPart;
"""

# outputs of the first part of the split algebra (the Ricci-dependent ones)
SPLIT_PART0 = ["At_rhs00", "At_rhs01", "At_rhs02", "At_rhs11", "At_rhs12", "At_rhs22"]
CUDA_SPLIT_OUT = os.path.join(REPO, "sympygr_b200", "csrc", "generated", "bssn_rhs_algebra_split.cuh")


def prune_stages(stages, outputs):
    """The staged capture restricted to the named outputs: the last stage keeps only
    those outputs, every earlier stage only the values something kept still reads
    (walked backwards from the outputs)."""
    out_name, out_defs = stages[-1]
    keep = [(n, e) for n, e in out_defs if str(n) in outputs]
    need = set()
    for _, e in keep:
        need |= e.free_symbols
    pruned = []
    for name, defs in reversed(stages[:-1]):
        kept = [(s, e) for s, e in defs if s in need]
        for _, e in kept:
            need |= e.free_symbols
        if kept:
            pruned.append((name, kept))
    pruned.reverse()
    pruned.append((out_name, keep))
    return pruned


def main_split(args):
    """The two-part algebra (bssn_rhs_algebra_split.cuh) from the staged capture."""
    from .staged import capture_staged

    CudaPrinter, _ = make_printers(src.load_dendro_c_printer(args.reference))
    slots = src.derivative_slots()
    stages = capture_staged(args.reference)
    if args.split_ricci:
        # the Ricci stage CSE'd in two halves (R00 R01 R02 / R11 R12 R22): a smaller
        # live set at the price of the subexpressions the halves share
        at = [i for i, st in enumerate(stages) if st[0] == "R"][0]
        defs = stages[at][1]
        stages = stages[:at] + [("R_a", defs[:3]), ("R_b", defs[3:])] + stages[at + 1:]
    parts = [SPLIT_PART0, [n for n in src.RHS_NAMES if n not in SPLIT_PART0]]
    texts, stats = [], {}
    for p, outs in enumerate(parts):
        body, nops, ntmp = emit_staged(prune_stages(stages, set(outs)), CudaPrinter(), slots)
        stats["nops%d" % p], stats["ntmp%d" % p] = nops, ntmp
        texts.append(
            "template <>\nstruct RhsAlgebraPart<%d> {\n"
            "  template <typename RT, class In, class Sink>\n"
            "  static __device__ __forceinline__ void run(const In& in, Sink& sink,\n"
            "                                             const AlgebraParams<RT>& prm, const RT eta) {\n"
            "%s\n  }\n};\n" % (p, "\n".join("  " + line for line in body)))
    with open(CUDA_SPLIT_OUT, "w") as f:
        f.write(CUDA_SPLIT_HEADER % stats)
        f.write("\n".join(texts))
        f.write("\n}  // namespace b200bssn\n")
    print("wrote", CUDA_SPLIT_OUT, stats)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the SymPyGR checkout")
    ap.add_argument("--split", action="store_true",
                    help="write only the two-part algebra (At_rhs / the rest) for the FP64 kernels")
    ap.add_argument("--split-ricci", action="store_true",
                    help="with --split: CSE the Ricci stage in two halves")
    ap.add_argument("--cache", default=None, help="optional pickle to reuse the CSE")
    ap.add_argument("--flat-cuda", action="store_true",
                    help="print the CUDA algebra from the single global CSE (as the C oracle)")
    ap.add_argument("--advective", action="store_true",
                    help="write only the upwind-mode algebra (advective derivatives in their own slots)")
    args = ap.parse_args(argv)
    if args.advective:
        return main_advective(args)
    if args.split:
        return main_split(args)

    t0 = time.time()
    if args.cache and os.path.exists(args.cache):
        with open(args.cache, "rb") as f:
            names, repl, reduced, orig = pickle.load(f)
    else:
        names, exprs = src.capture_bssn_rhs(args.reference)
        orig = sum(sp.count_ops(e) for e in exprs)
        repl, reduced = sp.cse(exprs, symbols=sp.numbered_symbols("t"), optimizations="basic")
        if args.cache:
            with open(args.cache, "wb") as f:
                pickle.dump((names, repl, reduced, orig), f)
    print("captured + cse: %.1fs, %d temporaries" % (time.time() - t0, len(repl)))

    CudaPrinter, CPrinter = make_printers(src.load_dendro_c_printer(args.reference))
    slots = src.derivative_slots()

    # constraints, flat (the oracle's C restatement): a fresh GR/constraints.py
    # import, before the staged capture turns dendro's geometry into symbols
    con_names, con_exprs = src.capture_constraints(args.reference)
    crepl, cred = sp.cse(con_exprs, symbols=sp.numbered_symbols("c"), optimizations="basic")
    cprog = schedule(con_names, crepl, cred)
    cbody, cnops = emit(cprog, CPrinter(), "c", slots, out_index=CON_INDEX)
    with open(C_CON_OUT, "w") as f:
        f.write(C_CON_HEADER)
        f.write("\n".join(cbody))
        f.write("\n}\n")
    prog = schedule(names, repl, reduced)

    if args.flat_cuda:
        body, nops = emit(prog, CudaPrinter(), "cuda", slots)
        ntmp = len(repl)
        header = CUDA_HEADER
    else:
        from .staged import capture_constraints_staged, capture_staged

        stages = capture_staged(args.reference)
        body, nops, ntmp = emit_staged(stages, CudaPrinter(), slots)
        header = CUDA_HEADER_STAGED
        # constraints: the RHS stages they use (not C3) + their own output stage
        con_stages = [st for st in stages if st[0] not in ("C3", "out")]
        con_stages += capture_constraints_staged(args.reference)
        cbody, cnops, _ = emit_staged(con_stages, CudaPrinter(), slots, out_index=CON_INDEX)
        with open(CUDA_CON_OUT, "w") as f:
            f.write(CUDA_CON_HEADER % {"nops": cnops})
            f.write("\n".join(cbody))
            f.write("\n}\n\n}  // namespace b200bssn\n")
    os.makedirs(os.path.dirname(CUDA_OUT), exist_ok=True)
    with open(CUDA_OUT, "w") as f:
        f.write(header % {"orig": orig, "nops": nops, "ntmp": ntmp})
        f.write("\n".join(body))
        f.write("\n}\n\n}  // namespace b200bssn\n")

    body, nops = emit(prog, CPrinter(), "c", slots)
    with open(C_OUT, "w") as f:
        f.write(C_HEADER % {"orig": orig, "nops": nops})
        f.write("\n".join(body))
        f.write("\n}\n")
    print("wrote", CUDA_OUT, "and", C_OUT)


if __name__ == "__main__":
    main()
