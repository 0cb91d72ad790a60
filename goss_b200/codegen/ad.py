"""Reverse-mode differentiation of a generated straight-line program.

Given the linearised program (``linear = d f_i / d y_i``, ``rhs = f``) this
builds its vector-Jacobian product: for cotangents ``abar`` (of ``linear``)
and ``bbar`` (of ``rhs``) it returns ``ybar = abar^T d(linear)/dy +
bbar^T d(rhs)/dy`` and the same with respect to the per-node field
parameters.  The adjoint of every assignment is emitted once, as the sum of
the contributions of the later statements that read it (SSA form), after a
forward sweep that recomputes the program's values:

    forward sweep:  v_j = f_j(inputs)                 (j = 1..J)
    outputs:        seeds abar_i, bbar_i
    reverse sweep:  a_j = sum_{k reads v_j} a_k * d f_k / d v_j   (j = J..1)
    results:        ybar_m = sum over statements reading state m, likewise F

With ``elementary=True`` (the default) the active statements are first split
so that every transcendental operation is a statement of its own: each
``exp(u)``, ``log(u)``, ``sqrt(u)``, ``u**p`` (p not an integer) and each
distinct factor of a denominator becomes a value ``__t<k>`` computed once in
the forward sweep, shared by all statements with the same operand (a
denominator ``d_1^2 d_2`` costs the reciprocals of ``d_1`` and ``d_2``, reused
by every other denominator containing them).  Their partial derivatives are
written in terms of those values -- d exp(u) = exp(u) du, d(1/d) = -(1/d)^2 dd,
d log(u) = (1/u) du, d sqrt(u) = du / (2 sqrt(u)) -- so the reverse sweep is
multiplications and additions only; the transcendental work of a VJP is that
of one forward evaluation.  Conditionals (``Piecewise``) are kept whole.

Partial derivatives of the remaining statements are sympy derivatives with
respect to their direct inputs (intermediates as independent symbols), with
floor derivatives 0 and |x|' = sign(x) as a Piecewise.
"""
from __future__ import annotations

from collections import defaultdict
from typing import Dict, List, Optional, Sequence, Set, Tuple

import sympy as sp

from .ir import CONST, STATE, TIME_CLS, Assign, Output, Program, clean


def _exp_shape(u: sp.Expr, active: Set[sp.Symbol]):
    """u = c0 + slope * mono with c0 a number and mono normalised so that the
    coefficient of its first term (in printed order) is 1: (shape key, slope,
    c0, mono), or None for an argument without state-dependent terms."""
    if not (u.free_symbols & active):
        return None
    c0, rest = u.as_coeff_Add()
    terms = []
    for t in sp.Add.make_args(rest):
        c, m = t.as_coeff_Mul()
        terms.append((str(m), float(c), m))
    terms.sort(key=lambda x: x[0])
    slope = terms[0][1]
    if slope == 0:
        return None
    key = tuple((name, round(c / slope, 12)) for name, c, _ in terms)
    mono = sp.Add(*[sp.Float(c / slope) * m if c != slope else m for _, c, m in terms])
    return key, slope, c0, mono


def _plan_exps(shapes: List[Tuple[tuple, float, sp.Expr]]) -> Dict:
    """Exponentials that share their argument's shape share one value:
    exp(c0 + s m) = e^c0 exp(s m), and exp(c0 + 2 s m) = e^c0 exp(s m)^2.
    Only shapes met with more than one distinct argument are planned."""
    args = defaultdict(set)
    for key, slope, c0 in shapes:
        args[key].add((slope, c0))
    plan = {}
    for key, members in args.items():
        if len(members) < 2:
            continue
        bases: List[float] = []
        for slope in sorted({sl for sl, _ in members}, key=abs):
            for b in bases:
                k = slope / b
                if abs(k - 2.0) < 1e-12:
                    plan[(key, slope)] = (b, 2)
                    break
            else:
                bases.append(slope)
                plan[(key, slope)] = (slope, 1)
    return plan


class _Splitter:
    """Rewrites active expressions so that transcendental operations are
    separate values (see the module docstring), recording their partials."""

    def __init__(self, active: Set[sp.Symbol], exp_plan: Optional[Dict] = None):
        self.active = active
        self.exp_plan = exp_plan                         # (argument shape, slope) -> (base slope, power)
        self.exp_args: List[Tuple[tuple, float, sp.Expr]] = []  # every exp argument's shape, slope, constant
        self.memo: Dict[sp.Expr, sp.Symbol] = {}
        self.nodes: List[Tuple[sp.Symbol, sp.Expr, Dict[sp.Symbol, sp.Expr]]] = []
        self.inverse_of: Dict[sp.Symbol, sp.Expr] = {}  # reciprocal value -> its base
        self.defs: Dict[sp.Symbol, sp.Expr] = {}        # split statement -> its expression
        self._count = 0

    def _is_active(self, e: sp.Expr) -> bool:
        return bool(e.free_symbols & self.active)

    def _node(self, expr: sp.Expr, partials) -> sp.Symbol:
        s = self.memo.get(expr)
        if s is not None:
            return s
        s = sp.Symbol(f"__t{self._count}", real=True)
        self._count += 1
        self.memo[expr] = s
        slot = len(self.nodes)
        self.nodes.append((s, expr, {}))
        self.active.add(s)
        self.nodes[slot] = (s, expr, partials(s))
        return s

    def _chain(self, outer: sp.Expr, u: sp.Expr) -> Dict[sp.Symbol, sp.Expr]:
        """{x: outer * du/dx} over the active symbols x of u."""
        out = {}
        for x in sorted(u.free_symbols & self.active, key=lambda q: q.name):
            d = clean(sp.diff(u, x))
            if d != 0:
                out[x] = outer * d
        return out

    def _free_inverse(self, e: sp.Expr, depth: int = 0):
        """1/e without a new reciprocal when e is a product of numbers,
        reciprocal values and statements defined that way (a gate's
        tau = alpha * beta with alpha = c/(1 + exp(u)) ...); else None."""
        if e.is_Number and e != 0:
            return 1 / e
        if e in self.inverse_of:
            return self.inverse_of[e]
        if isinstance(e, sp.Mul):
            parts = [self._free_inverse(f, depth) for f in e.args]
            return None if any(p is None for p in parts) else sp.Mul(*parts)
        if e.is_Pow and e.exp.is_Integer:
            inv = self._free_inverse(e.base, depth)
            return None if inv is None else inv ** e.exp
        if e.is_Symbol and e in self.defs and depth < 8:
            return self._free_inverse(self.defs[e], depth + 1)
        return None

    def recip_base(self, b: sp.Expr) -> sp.Expr:
        """1/b for one factor b: a value of its own, shared by every product
        and power of b (and 1/(1/x) = x)."""
        free = self._free_inverse(b)
        if free is not None:
            return free
        r = self._node(sp.Pow(b, -1, evaluate=False), lambda r: self._chain(-r * r, b))
        self.inverse_of.setdefault(r, b)
        return r

    def recip(self, d: sp.Expr) -> sp.Expr:
        """1/d for a product d of powers: the product of the reciprocals of its
        distinct bases, so each base costs one reciprocal however many
        denominators it appears in."""
        out = []
        for f in (d.args if isinstance(d, sp.Mul) else (d,)):
            if not self._is_active(f):
                out.append(sp.Pow(f, -1))
            elif f.is_Pow and f.exp.is_Integer and f.exp > 0:
                out.append(self.recip_base(f.base) ** f.exp)
            else:
                out.append(self.recip_base(f))
        return sp.Mul(*out)

    def exp(self, u: sp.Expr) -> sp.Expr:
        g = _exp_shape(u, self.active)
        if g is not None:
            key, slope, c0, mono = g
            self.exp_args.append((key, slope, c0))
            plan = (self.exp_plan or {}).get((key, slope))
            if plan is not None:
                base, power = plan
                arg = sp.Float(base) * mono
                e = self._node(sp.exp(arg), lambda e: self._chain(e, arg))
                return sp.Float(sp.N(sp.exp(c0), 20)) * e ** power
        return self._node(sp.exp(u), lambda e: self._chain(e, u))

    def log(self, u: sp.Expr) -> sp.Symbol:
        return self._node(sp.log(u), lambda l: self._chain(self.recip(u), u))

    def sqrt(self, u: sp.Expr) -> sp.Symbol:
        return self._node(sp.Pow(u, sp.Rational(1, 2), evaluate=False),
                          lambda s: self._chain(sp.Rational(1, 2) * self.recip(s), u))

    def power(self, b: sp.Expr, p: sp.Expr) -> sp.Symbol:
        """b**p with an inactive, non-integer exponent."""
        return self._node(sp.Pow(b, p, evaluate=False), lambda q: self._chain(p * q * self.recip(b), b))

    def _positive_power(self, b: sp.Expr, p: sp.Expr) -> sp.Expr:
        """Transformed b**p for an active base b and an inactive exponent p."""
        if p.is_Integer:
            return b ** p if p > 0 else self.recip(b ** (-p))
        if p == sp.Rational(1, 2):
            return self.sqrt(b)
        if p == sp.Rational(-1, 2):
            return self.recip(self.sqrt(b))
        return self.power(b, p)

    def tx(self, e: sp.Expr) -> sp.Expr:
        if e.is_Atom or not self._is_active(e) or isinstance(e, sp.Piecewise):
            return e
        if isinstance(e, sp.Mul):
            num, den = [], []
            for f in e.args:
                if f.is_Pow and self._is_active(f.base) and f.exp.is_Number and f.exp < 0:
                    den.append(self._positive_power(self.tx(f.base), -f.exp))
                else:
                    num.append(self.tx(f))
            if den:
                num.append(self.recip(sp.Mul(*den)))
            return sp.Mul(*num)
        if isinstance(e, sp.Pow):
            b, p = e.base, e.exp
            if b is sp.E:
                return self.exp(self.tx(p))
            if self._is_active(p):
                return e.func(self.tx(b), self.tx(p))
            if not self._is_active(b):
                return e
            return self._positive_power(self.tx(b), p)
        if isinstance(e, sp.exp):
            return self.exp(self.tx(e.args[0]))
        if isinstance(e, sp.log) and len(e.args) == 1:
            return self.log(self.tx(e.args[0]))
        return e.func(*[self.tx(a) for a in e.args])


class ReverseProgram:
    """Statements of the forward sweep and the reverse sweep.

    ``forward``: the forward sweep's assignments in order (with the split
    values when ``elementary``); ``outputs``: the program's outputs in terms
    of them; ``seeds``: (symbol, array, index) of the output cotangents;
    ``reverse``: (adjoint symbol, value) in evaluation order; ``state_bar`` and
    ``field_bar``: the VJP's results.  ``reverse=False`` builds the split
    forward program only.  With ``elementary`` a first pass over the program
    collects the exponentials' arguments, so that exponentials of the same
    shape share one value (``_plan_exps``).
    """

    def __init__(self, prog: Program, state_syms: Sequence[sp.Symbol], field_syms: Sequence[sp.Symbol],
                 inter_syms: Dict[str, sp.Symbol], elementary: bool = True, reverse: bool = True):
        self.state_syms = list(state_syms)
        self.field_syms = list(field_syms)
        plan = None
        if elementary:
            shapes = self._split_forward(prog, inter_syms, True, None)
            plan = _plan_exps(shapes)
        self._split_forward(prog, inter_syms, elementary, plan)
        self.seeds = []
        self.reverse: List[Tuple[sp.Symbol, sp.Expr]] = []
        if not reverse:  # the split forward program alone
            self.state_bar, self.field_bar = [], []
            return
        self._reverse_sweep()

    def _split_forward(self, prog: Program, inter_syms: Dict[str, sp.Symbol], elementary: bool,
                       plan: Optional[Dict]) -> List[Tuple[tuple, float, sp.Expr]]:
        """Fill forward / active_assigns / outputs; return the exp shapes met."""
        sym_of = dict(inter_syms)
        active: Set[sp.Symbol] = set(self.state_syms) | set(self.field_syms)
        splitter = _Splitter(active, plan) if elementary else None
        node_partials: Dict[sp.Symbol, Dict[sp.Symbol, sp.Expr]] = {}
        self.forward: List[Assign] = []
        self.active_assigns: List[Tuple[sp.Symbol, Assign]] = []

        def split(expr: sp.Expr, cls: int) -> sp.Expr:
            if splitter is None:
                return expr
            start = len(splitter.nodes)
            expr = splitter.tx(expr)
            for ns, ne, part in splitter.nodes[start:]:
                nb = Assign(ns.name, ne, cls)
                self.forward.append(nb)
                self.active_assigns.append((ns, nb))
                node_partials[ns] = part
            return expr

        for b in prog.body:
            if not isinstance(b, Assign):
                continue
            s = sym_of.get(b.name) or sp.Symbol(b.name, real=True)
            if b.cls in (CONST, TIME_CLS) or not (b.expr.free_symbols & active):
                self.forward.append(b)
                continue
            nb = Assign(b.name, split(b.expr, b.cls), b.cls)
            if splitter is not None:
                splitter.defs[s] = nb.expr
            active.add(s)
            self.forward.append(nb)
            self.active_assigns.append((s, nb))
        self.outputs: List[Output] = []
        for o in prog.body:
            if isinstance(o, Output):
                expr = split(o.expr, STATE) if (o.expr.free_symbols & active) else o.expr
                self.outputs.append(Output(o.array, o.index, expr))
        self.active = active
        self._node_partials = node_partials
        return splitter.exp_args if splitter is not None else []

    def _reverse_sweep(self) -> None:
        active, node_partials = self.active, self._node_partials
        # contributions[u] = adjoint-weighted partials of the statements reading u
        contrib: Dict[sp.Symbol, List[sp.Expr]] = defaultdict(list)
        for o in self.outputs:
            seed = sp.Symbol(f"__seed_{o.array}_{o.index}", real=True)
            self.seeds.append((seed, o.array, o.index))
            for u in sorted(o.expr.free_symbols & active, key=lambda q: q.name):
                d = clean(sp.diff(o.expr, u))
                if d != 0:
                    contrib[u].append(seed * d)
        for s, b in reversed(self.active_assigns):
            terms = contrib.pop(s, [])
            if not terms:
                continue
            adj = sp.Symbol(f"__adj_{s.name}", real=True)
            self.reverse.append((adj, sp.Add(*terms)))
            if s in node_partials:
                for u, d in node_partials[s].items():
                    contrib[u].append(adj * d)
                continue
            for u in sorted(b.expr.free_symbols & active, key=lambda q: q.name):
                d = clean(sp.diff(b.expr, u))
                if d != 0:
                    contrib[u].append(adj * d)
        self.state_bar = [sp.Add(*contrib.get(s, [])) for s in self.state_syms]
        self.field_bar = [sp.Add(*contrib.get(f, [])) for f in self.field_syms]
