"""Fold parameter-only sub-expressions into derived constants.

The device code evaluates the model millions of times per launch with the
same uniform parameters.  Every maximal sub-expression that depends on
uniform parameters only (``R*T/F``, ``1/(R*T)``, ``sqrt(K_o/5.4)``, ...) is
replaced by a *derived constant*: computed once per launch on the host in
FP64, passed in the kernel's parameter block (constant bank) next to the
parameters, and read by the kernel as a free operand.  Besides removing
arithmetic, this turns every division by a parameter-only expression into a
multiplication, which takes the reciprocals off the SFU pipe.

Groups of parameter-only factors inside a product (and terms inside a sum)
are folded as one constant, e.g. ``2*F*V_eff/(R*T)`` -> ``c*V_eff`` with
``c = 2*F/(R*T)``.  This re-associates a few operations relative to the
unfolded form; the results agree to rounding.
"""
from __future__ import annotations

from collections import OrderedDict
from typing import Dict, Iterable, List, Set, Tuple

import sympy as sp


class ConstantFolder:
    def __init__(self, uniform: Set[sp.Symbol], const_inter: Dict[sp.Symbol, sp.Expr]):
        self.uniform = set(uniform)
        self.const_inter = dict(const_inter)
        self.allowed = self.uniform | set(self.const_inter)
        self.table: "OrderedDict[str, Tuple[sp.Symbol, sp.Expr]]" = OrderedDict()

    # -- helpers -----------------------------------------------------------
    def is_const(self, e) -> bool:
        if isinstance(e, bool) or e in (sp.true, sp.false):
            return True
        fs = e.free_symbols
        return bool(fs) and fs <= self.allowed

    def slot(self, e: sp.Expr) -> sp.Symbol:
        key = sp.srepr(e)
        if key not in self.table:
            sym = sp.Symbol(f"__c{len(self.table)}", real=True)
            self.table[key] = (sym, e)
        return self.table[key][0]

    @property
    def derived(self) -> List[Tuple[sp.Symbol, sp.Expr]]:
        return list(self.table.values())

    # -- transform -----------------------------------------------------------
    def __call__(self, e):
        return self.t(e)

    def t(self, e):
        if isinstance(e, bool) or e in (sp.true, sp.false):
            return e
        if e.is_Number:
            return e
        if e.is_Symbol:
            return self.slot(e) if e in self.const_inter else e
        if self.is_const(e):
            return self.slot(e)
        if isinstance(e, (sp.Add, sp.Mul)):
            consts = [a for a in e.args if self.is_const(a)]
            nums = [a for a in e.args if a.is_Number]
            rest = [a for a in e.args if not self.is_const(a) and not a.is_Number]
            new_rest = [self.t(a) for a in rest]
            if consts and (len(consts) > 1 or nums or not (consts[0].is_Symbol and consts[0] in self.uniform)):
                c = self.slot(e.func(*(nums + consts)))
                return e.func(c, *new_rest)
            kept = nums + [self.t(a) for a in consts]
            return e.func(*(kept + new_rest))
        if isinstance(e, sp.Piecewise):
            return sp.Piecewise(*[(self.t(v), self.t(c)) for v, c in e.args], evaluate=False)
        if isinstance(e, sp.Pow):
            return sp.Pow(self.t(e.base), e.exp if e.exp.is_Number else self.t(e.exp))
        if isinstance(e, sp.core.relational.Relational):
            return e.func(self.t(e.lhs), self.t(e.rhs), evaluate=False)
        if isinstance(e, (sp.And, sp.Or)):
            return e.func(*[self.t(a) for a in e.args], evaluate=False)
        if isinstance(e, sp.Not):
            return sp.Not(self.t(e.args[0]))
        return e.func(*[self.t(a) for a in e.args])
