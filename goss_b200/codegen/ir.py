"""Straight-line programs derived from a parsed model.

A *program* is an ordered list of scalar assignments followed by writes to
output arrays.  Every target (the C restatement used by the oracle, the
goss C++ plugin class, the CUDA device code) is printed from the same
program, so all of them evaluate the same arithmetic in the same order.

Programs built here follow the generated-code contract of the reference:

* ``rhs``: ``ODE::eval(states, time, values)`` (reference
  ``python/goss/codegeneration.py:543-553``).
* ``linearized``: ``ODE::linearized_eval(states, time, linear, rhs,
  only_linear)`` (``codegeneration.py:584-620``): ``rhs = f(y, t)`` and
  ``linear[i] = d f_i / d y_i`` through all intermediates.  States whose
  ``f_i`` is linear in ``y_i`` (non-zero derivative free of ``y_i``) are
  flagged in ``linear_terms`` and computed before the ``only_linear`` early
  return; the remaining diagonal entries follow it (layout of
  ``cpp/tests/fhn.h:92-126`` and ``cpp/tests/beeler_reuter_1977.h:164-290``).

Each assignment carries a dependency class used by the GPU code:
``CONST`` (parameters only), ``FIELD`` (also per-node field parameters),
``TIME`` (time and parameters, no states) and ``STATE``.
"""
from __future__ import annotations

from collections import OrderedDict
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Set, Tuple

import sympy as sp

from .odeparse import TIME, ODEModel

CONST, FIELD, TIME_CLS, STATE = 0, 1, 2, 3
CLASS_NAMES = {CONST: "const", FIELD: "field", TIME_CLS: "time", STATE: "state"}


@dataclass
class Assign:
    name: str
    expr: sp.Expr
    cls: int = STATE


@dataclass
class Output:
    array: str
    index: int
    expr: sp.Expr


@dataclass
class Program:
    """Ordered assignments plus array outputs.

    ``split`` (optional) is the index into ``body`` at which the
    ``only_linear`` early return of ``linearized_eval`` sits: entries before
    it (assignments and outputs) are always evaluated.
    """

    name: str
    body: List[object] = field(default_factory=list)
    split: Optional[int] = None

    def assigns(self):
        return [b for b in self.body if isinstance(b, Assign)]

    def outputs(self):
        return [b for b in self.body if isinstance(b, Output)]


def _fix_derivative(expr: sp.Expr) -> sp.Expr:
    """Replace derivatives sympy leaves unevaluated by their values.

    ``floor``/``ceiling`` are piecewise constant, so their derivative is 0
    wherever it exists.
    """
    if not expr.has(sp.Derivative):
        return expr
    reps = {}
    for d in expr.atoms(sp.Derivative):
        if isinstance(d.expr, (sp.floor, sp.ceiling)):
            reps[d] = sp.Integer(0)
        else:
            raise ValueError(f"cannot differentiate {d.expr}")
    return expr.xreplace(reps)


def _sign_free(expr: sp.Expr) -> sp.Expr:
    # d|x|/dx = sign(x); keep it as a Piecewise so every printer handles it
    if not expr.has(sp.sign):
        return expr
    reps = {}
    for s in expr.atoms(sp.sign):
        a = s.args[0]
        reps[s] = sp.Piecewise((sp.Integer(1), a > 0), (sp.Integer(-1), a < 0), (sp.Integer(0), True))
    return expr.xreplace(reps)


def _heaviside_free(expr: sp.Expr) -> sp.Expr:
    if not expr.has(sp.Heaviside):
        return expr
    reps = {}
    for h in expr.atoms(sp.Heaviside):
        a = h.args[0]
        reps[h] = sp.Piecewise((sp.Integer(1), a > 0), (sp.Integer(0), True))
    return expr.xreplace(reps)


def clean(expr: sp.Expr) -> sp.Expr:
    return _heaviside_free(_sign_free(_fix_derivative(expr)))


class ModelIR:
    """Dependency analysis and programs for one model + field-parameter set."""

    def __init__(self, model: ODEModel, field_parameters: Sequence[str] = (),
                 field_states: Sequence[str] = (), monitored: Sequence[str] = (),
                 linearization: str = "gotran"):
        if linearization not in ("gotran", "exact"):
            raise ValueError("linearization must be 'gotran' or 'exact'")
        self.linearization = linearization
        self.model = model
        for p in field_parameters:
            if p not in model.parameters:
                raise ValueError(f"{p} is not a parameter in the {model.name} ODE")
        for s in field_states:
            if s not in model.states:
                raise ValueError(f"{s} is not a state in the {model.name} ODE")
        for m in monitored:
            if m not in model.intermediates:
                raise ValueError(f"{m} is not an expression in the {model.name} ODE")
        self.field_parameters = list(field_parameters)
        self.field_states = list(field_states)
        self.monitored = list(monitored)
        self.state_syms = [model.sym(s) for s in model.states]
        self.param_syms = [model.sym(p) for p in model.parameters]
        self.inter_syms = OrderedDict((k, model.sym(k)) for k in model.intermediates)
        self.inter_exprs: "OrderedDict[sp.Symbol, sp.Expr]" = OrderedDict(
            (model.sym(k), v) for k, v in model.intermediates.items())
        self.field_syms = {model.sym(p) for p in self.field_parameters}
        self._dclass_cache: Dict[sp.Symbol, int] = {}
        self._state_set = set(self.state_syms)
        self._param_set = set(self.param_syms)
        # transitive state dependencies of every intermediate
        self._deps: Dict[sp.Symbol, Set[sp.Symbol]] = {}
        self._cls: Dict[sp.Symbol, int] = {}
        for s, e in self.inter_exprs.items():
            self._deps[s] = self._expr_state_deps(e)
            self._cls[s] = self.expr_class(e)
        # derivative bookkeeping: (intermediate, state) -> symbol or expr
        self._dcache: Dict[Tuple[sp.Symbol, sp.Symbol], sp.Expr] = {}
        self._dassigns: "OrderedDict[sp.Symbol, sp.Expr]" = OrderedDict()

    # -- dependency helpers ------------------------------------------------
    def _expr_state_deps(self, e: sp.Expr) -> Set[sp.Symbol]:
        out: Set[sp.Symbol] = set()
        for s in e.free_symbols:
            if s in self._state_set:
                out.add(s)
            elif s in self._deps:
                out |= self._deps[s]
        return out

    def expr_class(self, e: sp.Expr) -> int:
        cls = CONST
        for s in e.free_symbols:
            if s in self._state_set:
                return STATE
            if s == TIME:
                cls = max(cls, TIME_CLS)
            elif s in self.field_syms:
                cls = max(cls, FIELD)
            elif s in self._cls:
                c = self._cls[s]
                if c == STATE:
                    return STATE
                cls = max(cls, c)
            elif s in self._dclass_cache:
                c = self._dclass_cache[s]
                if c == STATE:
                    return STATE
                cls = max(cls, c)
        # TIME combined with FIELD is still per node and time dependent
        return cls

    def depends_on(self, e: sp.Expr, y: sp.Symbol) -> bool:
        return y in self._expr_state_deps(e)

    # -- derivatives -------------------------------------------------------
    def total_derivative(self, e: sp.Expr, y: sp.Symbol) -> sp.Expr:
        """d e / d y with the chain rule through every intermediate.

        With ``linearization="gotran"`` the derivative reproduces what gotran
        generates for goss: when ``e`` contains ``y`` directly, its partial
        derivative already follows every intermediate ``k`` whose own
        expression contains ``y`` directly, and the chain rule then adds the
        path through ``k`` a second time.  The reference's generated
        Beeler-Reuter model shows this in ``linear[7]``
        (``cpp/tests/beeler_reuter_1977.h:265-286``: ``di_K1_dV`` contains
        ``dV_eff_1_dV`` and ``dV_eff_1_dV*di_K1_dV_eff_1`` is added again).
        ``"exact"`` counts every path once.
        """
        if not self.depends_on(e, y):
            return sp.Integer(0)
        inters = sorted(e.free_symbols & set(self.inter_exprs), key=lambda s: s.name)
        result = clean(sp.diff(e, y))
        if self.linearization == "gotran" and y in e.free_symbols:
            for k in inters:
                if y not in self.inter_exprs[k].free_symbols:
                    continue
                dk = self._dinter(k, y)
                part = clean(sp.diff(e, k))
                if dk != 0 and part != 0:
                    result = result + part * dk
        for k in inters:
            dk = self._dinter(k, y)
            if dk == 0:
                continue
            part = clean(sp.diff(e, k))
            if part == 0:
                continue
            result = result + part * dk
        return result

    def _dinter(self, k: sp.Symbol, y: sp.Symbol) -> sp.Expr:
        key = (k, y)
        if key in self._dcache:
            return self._dcache[key]
        if y not in self._deps[k]:
            self._dcache[key] = sp.Integer(0)
            return self._dcache[key]
        d = self.total_derivative(self.inter_exprs[k], y)
        if d.is_Number or d.is_Symbol:
            self._dcache[key] = d
            return d
        name = f"d{k.name}_d{y.name}"
        sym = sp.Symbol(name, real=True)
        self._dassigns[sym] = d
        self._dclass_cache[sym] = STATE
        self._dcache[key] = sym
        return sym

    # -- programs ------------------------------------------------------------
    def _needed_intermediates(self, exprs: Sequence[sp.Expr]) -> List[sp.Symbol]:
        need: Set[sp.Symbol] = set()
        stack = [s for e in exprs for s in e.free_symbols if s in self.inter_exprs]
        while stack:
            s = stack.pop()
            if s in need:
                continue
            need.add(s)
            stack.extend(t for t in self.inter_exprs[s].free_symbols if t in self.inter_exprs)
        return [s for s in self.inter_exprs if s in need]

    def rhs_program(self, result: str = "values") -> Program:
        m = self.model
        exprs = list(m.derivatives.values())
        prog = Program("rhs")
        for s in self._needed_intermediates(exprs):
            prog.body.append(Assign(s.name, self.inter_exprs[s], self._cls[s]))
        for i, e in enumerate(exprs):
            prog.body.append(Output(result, i, e))
        return prog

    def linear_terms(self) -> List[int]:
        self._linearize()
        return list(self._linear_flags)

    def _linearize(self):
        if hasattr(self, "_lin"):
            return
        lin = []
        flags = []
        for y, e in zip(self.state_syms, self.model.derivatives.values()):
            d = self.total_derivative(e, y)
            lin.append(d)
            # linear when the derivative is non-zero and does not involve y
            flags.append(int(d != 0 and not self._expr_dep_with_derivs(d, y)))
        self._lin = lin
        self._linear_flags = flags

    def _expr_dep_with_derivs(self, e: sp.Expr, y: sp.Symbol) -> bool:
        seen: Set[sp.Symbol] = set()
        stack = list(e.free_symbols)
        while stack:
            s = stack.pop()
            if s in seen:
                continue
            seen.add(s)
            if s == y:
                return True
            if s in self.inter_exprs:
                if y in self._deps[s]:
                    return True
            elif s in self._dassigns:
                stack.extend(self._dassigns[s].free_symbols)
        return False

    def _deriv_assign_order(self, roots: Sequence[sp.Expr]) -> List[sp.Symbol]:
        """Derivative intermediates needed by ``roots`` in dependency order."""
        order: List[sp.Symbol] = []
        seen: Set[sp.Symbol] = set()

        def visit(s):
            if s in seen or s not in self._dassigns:
                return
            seen.add(s)
            for t in sorted(self._dassigns[s].free_symbols, key=lambda q: q.name):
                visit(t)
            order.append(s)

        for r in roots:
            for s in sorted(r.free_symbols, key=lambda q: q.name):
                visit(s)
        return order

    def linearized_program(self, split: bool = True) -> Program:
        """``linearized_eval`` body: rhs, linear terms, then the rest."""
        self._linearize()
        m = self.model
        rhs = list(m.derivatives.values())
        prog = Program("linearized")
        lin_first = [i for i, f in enumerate(self._linear_flags) if f]
        lin_rest = [i for i, f in enumerate(self._linear_flags) if not f]
        # all plain intermediates needed by rhs or by any linear expression
        all_roots = rhs + self._lin + [self._dassigns[s] for s in self._dassigns]
        needed = self._needed_intermediates(all_roots)
        rhs_needed = set(self._needed_intermediates(rhs + [self._lin[i] for i in lin_first] +
                                                    [self._dassigns[s] for s in self._deriv_assign_order(
                                                        [self._lin[i] for i in lin_first])]))
        for s in needed:
            if s in rhs_needed:
                prog.body.append(Assign(s.name, self.inter_exprs[s], self._cls[s]))
        for i, e in enumerate(rhs):
            prog.body.append(Output("rhs", i, e))
        done: Set[sp.Symbol] = set()
        for s in self._deriv_assign_order([self._lin[i] for i in lin_first]):
            prog.body.append(Assign(s.name, self._dassigns[s], STATE))
            done.add(s)
        for i in lin_first:
            prog.body.append(Output("linear", i, self._lin[i]))
        prog.split = len(prog.body) if split else None
        for s in needed:
            if s not in rhs_needed:
                prog.body.append(Assign(s.name, self.inter_exprs[s], self._cls[s]))
        for s in self._deriv_assign_order([self._lin[i] for i in lin_rest]):
            if s not in done:
                prog.body.append(Assign(s.name, self._dassigns[s], STATE))
        for i in lin_rest:
            prog.body.append(Output("linear", i, self._lin[i]))
        if not split:
            prog.split = None
        return prog

    def jacobian_structure(self) -> List[List[bool]]:
        """``S[i][j]``: f_i depends on y_j through its expression or any
        intermediate it uses (a superset of the non-zero Jacobian entries; an
        entry outside it is exactly 0 in a forward-difference Jacobian too,
        since f_i is then computed from the same operands)."""
        out = []
        for e in self.model.derivatives.values():
            deps = self._expr_state_deps(e)
            out.append([y in deps for y in self.state_syms])
        return out

    def jacobian_program(self) -> Program:
        """``compute_jacobian(states, time, jac)`` body: ``jac[i*n + j] =
        d f_i / d y_j`` through every intermediate, each path counted once,
        every entry written (zeros too).

        The reference generates this override of ``ODE::compute_jacobian``
        (``cpp/goss/ODE.h:71``) when ``code_params["generate_jacobian"]`` is
        set (``python/goss/codegeneration.py:622-641``; gotran's
        ``jacobian_expressions``).  The derivatives here are exact whatever
        the linearisation rule of the diagonal in ``linearized``."""
        ex = self if self.linearization == "exact" else ModelIR(
            self.model, self.field_parameters, self.field_states, self.monitored, linearization="exact")
        m = self.model
        rhs = list(m.derivatives.values())
        n = len(self.state_syms)
        entries = [[ex.total_derivative(e, y) for y in self.state_syms] for e in rhs]
        roots = [d for row in entries for d in row]
        prog = Program("jacobian")
        for s in ex._needed_intermediates(roots + [ex._dassigns[s] for s in ex._deriv_assign_order(roots)]):
            prog.body.append(Assign(s.name, ex.inter_exprs[s], ex._cls[s]))
        for s in ex._deriv_assign_order(roots):
            prog.body.append(Assign(s.name, ex._dassigns[s], STATE))
        for i in range(n):
            for j in range(n):
                prog.body.append(Output("jac", i * n + j, entries[i][j]))
        return prog

    def monitored_program(self) -> Program:
        prog = Program("monitored")
        exprs = [self.inter_syms[k] for k in self.monitored]
        for s in self._needed_intermediates(exprs):
            prog.body.append(Assign(s.name, self.inter_exprs[s], self._cls[s]))
        for i, e in enumerate(exprs):
            prog.body.append(Output("monitored", i, e))
        return prog

    def class_of(self, name: str) -> int:
        s = self.model.symbols.get(name)
        if s is not None and s in self._cls:
            return self._cls[s]
        return STATE


def count_ops(prog: Program) -> Dict[str, int]:
    """Static operation census of a program (before compiler CSE).

    Classes: ``add`` (add/sub), ``mul``, ``div``, ``exp``, ``log``, ``sqrt``,
    ``pow``, ``cmp`` (comparisons/selects), ``misc`` (fabs/floor/...).
    Integer powers count as the multiplications a square-and-multiply chain
    needs.  Assignments in class CONST are excluded because they are loop
    invariant.
    """
    ops = dict(add=0, mul=0, div=0, exp=0, log=0, sqrt=0, pow=0, cmp=0, misc=0)

    def visit(e):
        if e.is_Atom:
            return
        if isinstance(e, sp.Add):
            ops["add"] += len(e.args) - 1
        elif isinstance(e, sp.Mul):
            num = [a for a in e.args if not (a.is_Pow and a.exp.is_Number and a.exp < 0)]
            den = [a for a in e.args if a.is_Pow and a.exp.is_Number and a.exp < 0]
            ops["mul"] += max(len(num) - 1, 0) + max(len(den) - 1, 0)
            if den:
                ops["div"] += 1
            for a in den:
                visit(sp.Pow(a.base, -a.exp))
            for a in num:
                visit(a)
            return
        elif isinstance(e, sp.Pow):
            ex = e.exp
            if ex.is_Integer:
                n = abs(int(ex))
                ops["mul"] += max(n.bit_length() - 1 + bin(n).count("1") - 1, 0)
                if ex < 0:
                    ops["div"] += 1
            elif ex == sp.Rational(1, 2):
                ops["sqrt"] += 1
            elif ex == sp.Rational(-1, 2):
                ops["sqrt"] += 1
                ops["div"] += 1
            else:
                ops["pow"] += 1
            visit(e.base)
            return
        elif isinstance(e, sp.exp):
            ops["exp"] += 1
        elif isinstance(e, sp.log):
            ops["log"] += 1
        elif isinstance(e, sp.Piecewise):
            ops["cmp"] += len(e.args) - 1
        elif isinstance(e, (sp.core.relational.Relational, sp.And, sp.Or, sp.Not)):
            ops["cmp"] += 1
        else:
            ops["misc"] += 1
        for a in e.args:
            visit(a)

    for b in prog.body:
        if isinstance(b, Assign):
            if b.cls == CONST:
                continue
            visit(b.expr)
        else:
            visit(b.expr)
    return ops
