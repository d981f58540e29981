"""CUDA printer backend for dendrosym's C code printer.

The reference prints its CSE'd algebra with ``DendroCPrinter``
(dendrosym/code_printer.py:9-158), a ``C99CodePrinter`` subclass that expands small
integer powers into products (``_print_Pow``, :44-72).  ``CudaPrinter`` extends it
for device code that is instantiated at more than one precision:

* every numeric constant is printed as a cast to the arithmetic type ``RT``
  (``((RT)0.6666666666666666)``), so the same text compiles to FP64 or FP32
  arithmetic without silent promotion of float expressions to double;
* integer powers are parenthesised products (the parent's bare ``x*x`` would
  print ``y/x**2`` as ``y/x*x``), negative powers become one division
  (``((RT)1)/((x*x))``), and ``x**(1/2)`` maps to ``sqrt``;
* symbols print as bare identifiers: the generator binds every input (state
  value, derivative, parameter) to a local of that name.

``CPrinter`` is the same with ``RT`` fixed to ``double``; it prints the oracle's
C restatement of the algebra.
"""
from __future__ import annotations

import sympy as sp
from sympy.printing.precedence import precedence


def make_printers(dendro_c_printer_cls):
    """Build (CudaPrinter, CPrinter) on top of the reference's DendroCPrinter."""

    class CudaPrinter(dendro_c_printer_cls):
        """Typed-constant CUDA printer (see module docstring)."""

        def __init__(self, rt: str = "RT"):
            super().__init__()
            self.rt = rt

        # ---- numbers -------------------------------------------------------
        def _typed(self, v: float) -> str:
            return "((%s)%r)" % (self.rt, float(v))

        def _print_Integer(self, expr):
            return "((%s)%d)" % (self.rt, int(expr))

        def _print_Rational(self, expr):
            return self._typed(float(expr))

        def _print_Float(self, expr):
            return self._typed(float(expr))

        def _print_Half(self, expr):
            return self._typed(0.5)

        def _print_NegativeOne(self, expr):
            return "((%s)-1)" % self.rt

        def _print_One(self, expr):
            return "((%s)1)" % self.rt

        def _print_Zero(self, expr):
            return "((%s)0)" % self.rt

        # ---- powers --------------------------------------------------------
        def _print_Pow(self, expr):
            prec = precedence(expr)
            base, ex = expr.base, expr.exp
            if ex.is_Integer:
                n = int(ex)
                if 2 <= n <= 6:
                    # parenthesised: the product may stand in a denominator,
                    # where a bare x*x would read as (1/x)*x
                    return "(%s)" % "*".join([self.parenthesize(base, prec)] * n)
                if -6 <= n <= -1:
                    return "((%s)1)/(%s)" % (
                        self.rt,
                        "*".join([self.parenthesize(base, prec)] * (-n)),
                    )
            if ex == sp.Rational(1, 2):
                return "sqrt(%s)" % self._print(base)
            if ex == sp.Rational(-1, 2):
                return "((%s)1)/sqrt(%s)" % (self.rt, self._print(base))
            return "pow(%s, %s)" % (self._print(base), self._print(ex))

        def _print_Symbol(self, expr):
            return expr.name

    class CPrinter(CudaPrinter):
        """Plain C99 flavour with double arithmetic (oracle)."""

        def __init__(self):
            super().__init__(rt="double")

    return CudaPrinter, CPrinter
