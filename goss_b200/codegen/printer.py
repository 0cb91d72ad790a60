"""Print sympy expression trees as C-family source.

One printer serves the C restatement (oracle), the goss C++ plugin class
and the CUDA device code.  It never re-associates: ``a + b + c`` is printed
``((a + b) + c)`` exactly as the sympy tree is ordered, so every target
performs the same floating-point operations in the same order.

Conventions:

* Rational coefficients print as a single literal multiplier
  (``x/7`` becomes ``0.14285714285714285*x``).
* Positive integer powers print as explicit products built by repeated
  squaring; negative powers become a division.
* ``Pow(x, 1/2)`` prints ``sqrt``; other real exponents print ``pow``.
* ``Piecewise`` prints nested ``?:``.
"""
from __future__ import annotations

from typing import Callable, Dict, Optional

import sympy as sp


_LOG2E = 1.4426950408889634  # log2(e)


def c_double(v: float) -> str:
    r = repr(float(v))
    if r in ("inf", "-inf", "nan"):
        raise ValueError(f"non-finite constant {r}")
    if "e" not in r and "." not in r:
        r += ".0"
    return r


class CPrinter:
    """Configurable C/C++/CUDA expression printer.

    ``sym`` maps a sympy Symbol to its source text.  ``fn`` maps function
    names (``exp``, ``log``, ``sqrt``, ``fabs``, ``floor``, ``ceil``, ``pow``,
    ``fmax``, ``fmin``, ``sin``...) to the callee name of the target.
    ``lit`` formats a numeric constant.
    """

    def __init__(self, sym: Callable[[sp.Symbol], str], fn: Optional[Dict[str, str]] = None,
                 lit: Callable[[float], str] = c_double, exp2_fold: bool = False):
        self.sym = sym
        # exp(c*x) with a numeric c printed as exp2((c*log2(e))*x): the
        # hardware exponential is base 2, so this saves the multiply by log2(e)
        self.exp2_fold = exp2_fold
        self.fn = dict(exp="exp", exp2="exp2", log="log", sqrt="sqrt", fabs="fabs", floor="floor", ceil="ceil",
                       pow="pow", fmax="fmax", fmin="fmin", sin="sin", cos="cos", tan="tan", tanh="tanh")
        if fn:
            self.fn.update(fn)
        self.lit = lit

    # -- helpers -----------------------------------------------------------
    def _f(self, name: str, *args: str) -> str:
        return f"{self.fn[name]}({', '.join(args)})"

    def _ipow(self, base: str, n: int) -> str:
        """x**n, n >= 1, as products (square and multiply)."""
        if n == 1:
            return base
        if n == 2:
            return f"({base}*{base})"
        if n == 3:
            return f"({base}*{base}*{base})"
        half = self._ipow(base, n // 2)
        sq = f"({half}*{half})"
        return sq if n % 2 == 0 else f"({sq}*{base})"

    # -- main entry ---------------------------------------------------------
    def __call__(self, e) -> str:
        return self.p(e)

    def p(self, e) -> str:
        if isinstance(e, bool) or e is sp.true or e is sp.false:
            return "1" if bool(e) else "0"
        if e.is_Symbol:
            return self.sym(e)
        if e.is_Number:
            v = float(e)
            s = self.lit(abs(v))
            return f"(-{s})" if v < 0 else s
        if e is sp.pi:
            return self.lit(float(sp.pi))
        if isinstance(e, sp.Add):
            return "(" + " + ".join(self.p(a) for a in e.args).replace("+ (-", "- (") + ")"
        if isinstance(e, sp.Mul):
            return self._mul(e)
        if isinstance(e, sp.Pow):
            return self._pow(e)
        if isinstance(e, sp.exp):
            return self._exp(e.args[0])
        if isinstance(e, sp.log):
            if len(e.args) != 1:
                raise ValueError("log with base is not supported")
            return self._f("log", self.p(e.args[0]))
        if isinstance(e, sp.Abs):
            return self._f("fabs", self.p(e.args[0]))
        if isinstance(e, sp.floor):
            return self._f("floor", self.p(e.args[0]))
        if isinstance(e, sp.ceiling):
            return self._f("ceil", self.p(e.args[0]))
        if isinstance(e, (sp.sin, sp.cos, sp.tan, sp.tanh)):
            return self._f(type(e).__name__, self.p(e.args[0]))
        if isinstance(e, sp.Max):
            out = self.p(e.args[0])
            for a in e.args[1:]:
                out = self._f("fmax", out, self.p(a))
            return out
        if isinstance(e, sp.Min):
            out = self.p(e.args[0])
            for a in e.args[1:]:
                out = self._f("fmin", out, self.p(a))
            return out
        if isinstance(e, sp.Piecewise):
            return self._piecewise(e.args)
        if isinstance(e, sp.core.relational.Relational):
            op = {"<": "<", "<=": "<=", ">": ">", ">=": ">=", "==": "==", "!=": "!="}[e.rel_op]
            return f"({self.p(e.lhs)} {op} {self.p(e.rhs)})"
        if isinstance(e, sp.And):
            return "(" + " && ".join(self.p(a) for a in e.args) + ")"
        if isinstance(e, sp.Or):
            return "(" + " || ".join(self.p(a) for a in e.args) + ")"
        if isinstance(e, sp.Not):
            return f"(!{self.p(e.args[0])})"
        raise ValueError(f"cannot print {type(e).__name__}: {e}")

    def _exp(self, arg) -> str:
        if self.exp2_fold:
            c, rest = arg.as_coeff_Mul()
            if c.is_Number and c != 1 and rest != 1:
                return self._f("exp2", f"{self.lit(float(c) * _LOG2E)}*{self.p(rest)}"
                               if float(c) > 0 else f"(-{self.lit(-float(c) * _LOG2E)})*{self.p(rest)}")
        return self._f("exp", self.p(arg))

    def _piecewise(self, pieces) -> str:
        (val, cond), rest = pieces[0], pieces[1:]
        if cond is sp.true or cond == True:  # noqa: E712
            return self.p(val)
        if not rest:
            # no otherwise branch: goss/gotran semantics are undefined there;
            # emit 0 like a missing value
            return f"({self.p(cond)} ? {self.p(val)} : {self.lit(0.0)})"
        return f"({self.p(cond)} ? {self.p(val)} : {self._piecewise(rest)})"

    def _pow(self, e: sp.Pow) -> str:
        b, x = e.base, e.exp
        if b is sp.E:
            return self._exp(x)
        if x.is_Integer:
            n = int(x)
            if n == 0:
                return self.lit(1.0)
            if n > 0:
                return self._ipow(self.p(b), n)
            return f"({self.lit(1.0)}/{self._ipow(self.p(b), -n)})"
        if x == sp.Rational(1, 2):
            return self._f("sqrt", self.p(b))
        if x == sp.Rational(-1, 2):
            return f"({self.lit(1.0)}/{self._f('sqrt', self.p(b))})"
        return self._f("pow", self.p(b), self.p(x))

    def _mul(self, e: sp.Mul) -> str:
        coeff, factors = e.as_coeff_mul()
        num, den = [], []
        for f in factors:
            if f.is_Pow and f.exp.is_Number and f.exp < 0:
                inv = sp.Pow(f.base, -f.exp)
                den.append(self.p(inv))
            else:
                num.append(self.p(f))
        neg = False
        c = float(coeff)
        if c < 0:
            neg = True
            c = -c
        parts = []
        if c != 1.0 or not num:
            parts.append(self.lit(c))
        parts.extend(num)
        s = "*".join(parts)
        if den:
            d = "*".join(den)
            s = f"{s}/({d})" if len(den) > 1 else f"{s}/{d}"
        s = f"({s})"
        return f"(-{s})" if neg else s
