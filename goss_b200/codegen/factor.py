"""Greedy common-factor extraction for printed sums (fewer multiplications).

Sympy keeps sums of products expanded: ``0.06*V - 0.06*E_K`` or
``a*b*x + a*c*y + a*z`` cost one multiplication per term and factor.  For
every sum, :func:`factor_common` repeatedly pulls out the factor (a symbol,
a power's base or a numeric coefficient's magnitude) that the most terms
share -- ``0.06*(V - E_K)``, ``a*(b*x + c*y + z)`` -- and recurses into the
groups.  The result is the same value in exact arithmetic; rounding differs,
so the pass is applied only to the forms whose arithmetic order is free (the
FP32 kernels' split model and the reverse-mode sweeps), never to the FP64
programs that reproduce the reference's operations.  Products are built
unevaluated so that sympy does not distribute a number back over the sum.
"""
from __future__ import annotations

from collections import Counter
from typing import Dict, List, Tuple

import sympy as sp

_NUM = "#num"


def _term_factors(t: sp.Expr) -> Tuple[sp.Expr, Dict[sp.Expr, int]]:
    """(numeric coefficient, {base: positive integer power}) of a product term."""
    c, rest = t.as_coeff_Mul()
    f: Dict[sp.Expr, int] = {}
    for a in sp.Mul.make_args(rest):
        b, p = a.as_base_exp()
        if p.is_Integer and p > 0:
            f[b] = f.get(b, 0) + int(p)
        else:
            f[a] = f.get(a, 0) + 1
    return c, f


def _rebuild(c: sp.Expr, f: Dict[sp.Expr, int]) -> sp.Expr:
    parts = [b ** p if p != 1 else b for b, p in f.items() if p > 0]
    if not parts:
        return c
    body = sp.Mul(*parts)
    return body if c == 1 else (-body if c == -1 else sp.Mul(c, body, evaluate=False))


def _fold_add(terms: List[sp.Expr]) -> sp.Expr:
    if len(terms) < 2:
        return sp.Add(*terms)
    info = [_term_factors(t) for t in terms]
    count: Counter = Counter()
    for c, f in info:
        for b in f:
            count[b] += 1
        if c.is_Number and abs(c) != 1:
            count[(_NUM, abs(c))] += 1
    if not count:
        return sp.Add(*terms)
    best, n = max(count.items(), key=lambda kv: (kv[1], not isinstance(kv[0], tuple), str(kv[0])))
    if n < 2:
        return sp.Add(*terms)
    inside, outside = [], []
    for (c, f), t in zip(info, terms):
        if isinstance(best, tuple):
            if c.is_Number and abs(c) == best[1]:
                inside.append(_rebuild(sp.Integer(1) if c > 0 else sp.Integer(-1), f))
                continue
        elif best in f:
            g = dict(f)
            g[best] -= 1
            inside.append(_rebuild(c, g))
            continue
        outside.append(t)
    factor = best[1] if isinstance(best, tuple) else best
    prod = sp.Mul(factor, _fold_add(inside), evaluate=False)
    if not outside:
        return prod
    return sp.Add(prod, _fold_add(outside), evaluate=False)


def factor_common(e: sp.Expr) -> sp.Expr:
    """``e`` with common factors pulled out of every sum (see module doc)."""
    if e.is_Atom or isinstance(e, (sp.core.relational.Relational, sp.logic.boolalg.Boolean)):
        return e
    if isinstance(e, sp.Piecewise):
        return sp.Piecewise(*[(factor_common(v), c) for v, c in e.args], evaluate=False)
    args = [factor_common(a) for a in e.args]
    if isinstance(e, sp.Add):
        return _fold_add(list(sp.Add.make_args(sp.Add(*args))))
    if isinstance(e, sp.Mul):
        return sp.Mul(*args, evaluate=False)
    return e.func(*args)
