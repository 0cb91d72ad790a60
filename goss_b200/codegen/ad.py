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

Partial derivatives are sympy derivatives of each statement with respect to
its direct inputs (intermediates as independent symbols), with floor
derivatives 0 and |x|' = sign(x) as a Piecewise.
"""
from __future__ import annotations

from collections import OrderedDict, defaultdict
from typing import Dict, List, Sequence, Set, Tuple

import sympy as sp

from .ir import CONST, TIME_CLS, Assign, Output, Program, clean


class ReverseProgram:
    """Statements of the forward sweep and the reverse sweep."""

    def __init__(self, prog: Program, state_syms: Sequence[sp.Symbol], field_syms: Sequence[sp.Symbol],
                 inter_syms: Dict[str, sp.Symbol]):
        self.forward: List[Assign] = [b for b in prog.body if isinstance(b, Assign)]
        outputs = [b for b in prog.body if isinstance(b, Output)]
        self.state_syms = list(state_syms)
        self.field_syms = list(field_syms)
        sym_of = dict(inter_syms)
        active: Set[sp.Symbol] = set(self.state_syms) | set(self.field_syms)
        self.active_assigns: List[Tuple[sp.Symbol, Assign]] = []
        for b in self.forward:
            s = sym_of.get(b.name) or sp.Symbol(b.name, real=True)
            if b.cls in (CONST, TIME_CLS):
                continue
            if b.expr.free_symbols & active:
                active.add(s)
                self.active_assigns.append((s, b))
        self.active = active
        # contributions[u] = list of (adjoint expression, partial expression)
        contrib: Dict[sp.Symbol, List[sp.Expr]] = defaultdict(list)
        self.seeds = []
        for o in outputs:
            seed = sp.Symbol(f"__seed_{o.array}_{o.index}", real=True)
            self.seeds.append((seed, o.array, o.index))
            for u in sorted(o.expr.free_symbols & active, key=lambda q: q.name):
                d = clean(sp.diff(o.expr, u))
                if d != 0:
                    contrib[u].append(seed * d)
        self.reverse: List[Tuple[sp.Symbol, sp.Expr]] = []  # (adjoint symbol, value)
        for s, b in reversed(self.active_assigns):
            terms = contrib.pop(s, [])
            if not terms:
                continue
            adj = sp.Symbol(f"__adj_{s.name}", real=True)
            self.reverse.append((adj, sp.Add(*terms)))
            for u in sorted(b.expr.free_symbols & active, key=lambda q: q.name):
                d = clean(sp.diff(b.expr, u))
                if d != 0:
                    contrib[u].append(adj * d)
        self.state_bar = [sp.Add(*contrib.get(s, [])) for s in self.state_syms]
        self.field_bar = [sp.Add(*contrib.get(f, [])) for f in self.field_syms]
