"""Front end for gotran ``.ode`` model files.

gotran (the third-party package goss uses to read ``.ode`` files,
``python/goss/ode.py:1-30`` and ``python/goss/compilemodule.py:85-117`` in the
reference) is not available, so this module reads the same DSL itself.  A
``.ode`` file is syntactically Python; it is parsed with :mod:`ast` and never
executed.  The subset understood here is the one the cardiac cell models in
the reference use:

* ``parameters("Component", ..., name=value | ScalarParam(value, ...))``
* ``states("Component", ..., name=value | ScalarParam(value, ...))``
* ``expressions("Component", ...)`` / ``component(...)`` / ``comment(...)``
* ``name = expr`` (intermediate) and ``dX_dt = expr`` (time derivative of X)
* ``exp log sqrt abs floor ceil sin cos tan tanh``, ``**``, ``time``
* ``Conditional(cond, a, b)``, ``ContinuousConditional(cond, a, b, sigma)``
  with ``Lt Le Gt Ge Eq Ne And Or Not`` conditions.

Ordering follows gotran, which goss exposes unchanged through ``state_names``
/ ``parameter_names`` (reference ``tests/test_ode_bindings.py:123-131``):
states are numbered in the order their ``dX_dt`` is defined, and the
parameters of each ``parameters(...)`` declaration are sorted by name.
"""
from __future__ import annotations

import ast
import math
from collections import OrderedDict
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Tuple

import sympy as sp


class ODEParseError(ValueError):
    """Raised for ``.ode`` input outside the supported subset."""


# ---------------------------------------------------------------------------
# Relational / logical helpers kept as plain sympy objects
# ---------------------------------------------------------------------------
_REL = {
    "Lt": sp.StrictLessThan,
    "Le": sp.LessThan,
    "Gt": sp.StrictGreaterThan,
    "Ge": sp.GreaterThan,
    "Eq": sp.Eq,
    "Ne": sp.Ne,
}

_FUNCS = {
    "exp": sp.exp,
    "log": sp.log,
    "sqrt": sp.sqrt,
    "abs": sp.Abs,
    "Abs": sp.Abs,
    "floor": sp.floor,
    "ceil": sp.ceiling,
    "sin": sp.sin,
    "cos": sp.cos,
    "tan": sp.tan,
    "tanh": sp.tanh,
}

TIME = sp.Symbol("time", real=True)


def _num(value) -> sp.Expr:
    if isinstance(value, bool):
        return sp.Integer(int(value))
    if isinstance(value, int):
        return sp.Integer(value)
    if isinstance(value, float):
        if value == int(value) and abs(value) < 2**52:
            # keep integral floats exact (``40.`` and ``40`` mean the same)
            return sp.Integer(int(value))
        return sp.Float(value)
    raise ODEParseError(f"unsupported literal {value!r}")


def continuous_conditional(cond, true_value, false_value, sigma) -> sp.Expr:
    """Smooth step used by gotran for ``ContinuousConditional``.

    ``Ge/Gt(x, y)`` becomes the logistic ``1 - 1/(1 + exp((x - y)/sigma))`` and
    ``Le/Lt(x, y)`` becomes ``1/(1 + exp((x - y)/sigma))``; this is the form
    the reference's generated FitzHugh-Nagumo model carries
    (``cpp/tests/fhn.h:83-85`` generated from ``cpp/tests/fhn.ode:27``).
    """
    if not isinstance(cond, sp.core.relational.Relational):
        raise ODEParseError("ContinuousConditional needs a single relational condition")
    x, y = cond.lhs, cond.rhs
    z = (x - y) / sigma
    if isinstance(cond, (sp.StrictGreaterThan, sp.GreaterThan)):
        step = 1 - 1 / (1 + sp.exp(z))
    elif isinstance(cond, (sp.StrictLessThan, sp.LessThan)):
        step = 1 / (1 + sp.exp(z))
    else:
        raise ODEParseError("ContinuousConditional supports Lt/Le/Gt/Ge only")
    return false_value + (true_value - false_value) * step


@dataclass
class ODEModel:
    """Parsed model: declaration-ordered states, parameters and expressions."""

    name: str
    states: "OrderedDict[str, float]" = field(default_factory=OrderedDict)
    parameters: "OrderedDict[str, float]" = field(default_factory=OrderedDict)
    # intermediates in definition order: name -> sympy expression
    intermediates: "OrderedDict[str, sp.Expr]" = field(default_factory=OrderedDict)
    # state name -> expression of its time derivative
    derivatives: "OrderedDict[str, sp.Expr]" = field(default_factory=OrderedDict)
    components: Dict[str, str] = field(default_factory=dict)
    symbols: Dict[str, sp.Symbol] = field(default_factory=dict)
    source: Optional[str] = None

    # -- convenience -----------------------------------------------------
    @property
    def state_names(self) -> List[str]:
        return list(self.states)

    @property
    def parameter_names(self) -> List[str]:
        return list(self.parameters)

    @property
    def num_states(self) -> int:
        return len(self.states)

    @property
    def num_parameters(self) -> int:
        return len(self.parameters)

    def sym(self, name: str) -> sp.Symbol:
        return self.symbols[name]

    @property
    def is_dae(self) -> bool:
        return False

    def signature(self) -> str:
        """Stable text form of the model used for cache keys."""
        parts = [self.name]
        parts += [f"s:{k}={v!r}" for k, v in self.states.items()]
        parts += [f"p:{k}={v!r}" for k, v in self.parameters.items()]
        parts += [f"i:{k}={sp.srepr(v)}" for k, v in self.intermediates.items()]
        parts += [f"d:{k}={sp.srepr(v)}" for k, v in self.derivatives.items()]
        return "\n".join(parts)


class _Builder:
    def __init__(self, name: str):
        self.model = ODEModel(name=name)
        self.component = ""
        self.pending_derivs: List[Tuple[str, ast.AST]] = []

    # -- symbols -----------------------------------------------------------
    def _new_symbol(self, name: str) -> sp.Symbol:
        if name in self.model.symbols:
            raise ODEParseError(f"'{name}' is declared twice")
        if name == "time" or name == "t" and False:
            raise ODEParseError("'time' is reserved")
        s = sp.Symbol(name, real=True)
        self.model.symbols[name] = s
        return s

    def _value(self, node: ast.AST, what: str) -> float:
        """Numeric default of a ``name=...`` keyword in parameters()/states()."""
        if isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id == "ScalarParam":
            if not node.args:
                raise ODEParseError(f"ScalarParam without value for {what}")
            node = node.args[0]
        try:
            value = ast.literal_eval(node)
        except Exception:
            # allow simple constant arithmetic such as -85.0 or 1e-3*2
            expr = self.expr(node, allow_symbols=False)
            value = float(expr)
        if isinstance(value, bool) or not isinstance(value, (int, float)):
            raise ODEParseError(f"non-numeric default for {what}")
        return float(value)

    # -- expressions ---------------------------------------------------------
    def expr(self, node: ast.AST, allow_symbols: bool = True) -> sp.Expr:
        e = self.expr
        if isinstance(node, ast.Constant):
            if isinstance(node.value, (int, float)) and not isinstance(node.value, bool):
                return _num(node.value)
            raise ODEParseError(f"unsupported constant {node.value!r}")
        if isinstance(node, ast.Name):
            if not allow_symbols:
                raise ODEParseError(f"symbol '{node.id}' not allowed here")
            if node.id == "time":
                return TIME
            if node.id == "pi":
                return sp.pi
            if node.id in self.model.symbols:
                return self.model.symbols[node.id]
            raise ODEParseError(f"'{node.id}' used before it is defined")
        if isinstance(node, ast.UnaryOp):
            if isinstance(node.op, ast.USub):
                return -e(node.operand, allow_symbols)
            if isinstance(node.op, ast.UAdd):
                return e(node.operand, allow_symbols)
            if isinstance(node.op, ast.Not):
                return sp.Not(e(node.operand, allow_symbols))
        if isinstance(node, ast.BinOp):
            a, b = e(node.left, allow_symbols), e(node.right, allow_symbols)
            if isinstance(node.op, ast.Add):
                return a + b
            if isinstance(node.op, ast.Sub):
                return a - b
            if isinstance(node.op, ast.Mult):
                return a * b
            if isinstance(node.op, ast.Div):
                return a / b
            if isinstance(node.op, ast.Pow):
                return a**b
        if isinstance(node, ast.Call) and isinstance(node.func, ast.Name):
            fname = node.func.id
            args = [e(a, allow_symbols) for a in node.args]
            if node.keywords:
                raise ODEParseError(f"keyword arguments to {fname} are not supported")
            if fname in _FUNCS:
                if len(args) != 1:
                    raise ODEParseError(f"{fname} takes one argument")
                return _FUNCS[fname](args[0])
            if fname in ("pow",):
                return args[0] ** args[1]
            if fname in _REL:
                if len(args) != 2:
                    raise ODEParseError(f"{fname} takes two arguments")
                return _REL[fname](args[0], args[1], evaluate=False)
            if fname == "And":
                return sp.And(*args, evaluate=False)
            if fname == "Or":
                return sp.Or(*args, evaluate=False)
            if fname == "Not":
                return sp.Not(args[0])
            if fname == "Conditional":
                if len(args) != 3:
                    raise ODEParseError("Conditional takes (cond, true, false)")
                return sp.Piecewise((args[1], args[0]), (args[2], True), evaluate=False)
            if fname == "ContinuousConditional":
                if len(args) != 4:
                    raise ODEParseError("ContinuousConditional takes (cond, true, false, sigma)")
                return continuous_conditional(*args)
            if fname in ("Max", "max"):
                return sp.Max(*args)
            if fname in ("Min", "min"):
                return sp.Min(*args)
            raise ODEParseError(f"unsupported function '{fname}'")
        raise ODEParseError(f"unsupported syntax: {ast.dump(node)[:80]}")

    # -- statements ------------------------------------------------------------
    def statement(self, st: ast.stmt) -> None:
        if isinstance(st, ast.Expr) and isinstance(st.value, ast.Constant):
            return  # docstring-like literal
        if isinstance(st, ast.Expr) and isinstance(st.value, ast.Call) and isinstance(st.value.func, ast.Name):
            call = st.value
            kind = call.func.id
            comps = []
            for a in call.args:
                try:
                    comps.append(str(ast.literal_eval(a)))
                except Exception as exc:  # pragma: no cover - malformed input
                    raise ODEParseError(f"{kind}(): positional arguments must be strings") from exc
            if kind in ("parameters", "states"):
                comp = comps[0] if comps else self.component
                keywords = list(call.keywords)
                if kind == "parameters":
                    # gotran orders the parameters of one declaration by name
                    # (e.g. K_mNa, K_mk, P_NaK in the generated TP06 code,
                    # reference benchmarks/tentusscher_panfilov_2006_M_cell.py:37-90)
                    keywords.sort(key=lambda kw: kw.arg or "")
                for kw in keywords:
                    if kw.arg is None:
                        raise ODEParseError(f"**kwargs not supported in {kind}()")
                    value = self._value(kw.value, kw.arg)
                    self._new_symbol(kw.arg)
                    target = self.model.parameters if kind == "parameters" else self.model.states
                    target[kw.arg] = value
                    self.model.components[kw.arg] = comp
                return
            if kind in ("expressions", "component"):
                self.component = comps[0] if comps else ""
                return
            if kind in ("comment", "model_arguments"):
                return
            raise ODEParseError(f"unsupported declaration '{kind}'")
        if isinstance(st, ast.Assign):
            if len(st.targets) != 1 or not isinstance(st.targets[0], ast.Name):
                raise ODEParseError("only 'name = expression' assignments are supported")
            name = st.targets[0].id
            value = self.expr(st.value)
            if name.startswith("d") and name.endswith("_dt") and name[1:-3] in self.model.states:
                state = name[1:-3]
                if state in self.model.derivatives:
                    raise ODEParseError(f"derivative of '{state}' given twice")
                self.model.derivatives[state] = value
                self.model.components[name] = self.component
                return
            sym = self._new_symbol(name)
            self.model.intermediates[name] = value
            self.model.components[name] = self.component
            del sym
            return
        raise ODEParseError(f"unsupported statement at line {getattr(st, 'lineno', '?')}")


def parse_ode_text(text: str, name: str) -> ODEModel:
    """Parse ``.ode`` source text into an :class:`ODEModel`."""
    try:
        tree = ast.parse(text)
    except SyntaxError as exc:
        raise ODEParseError(f"{name}: {exc}") from exc
    b = _Builder(name)
    for st in tree.body:
        b.statement(st)
    m = b.model
    missing = [s for s in m.states if s not in m.derivatives]
    if missing:
        # goss only supports algebraic states through DAE solvers, which are
        # outside the multi-node GPU path
        raise ODEParseError(f"{name}: no time derivative for state(s) {missing} (DAEs are not supported)")
    # gotran numbers the states in the order their time derivatives are
    # defined (cpp/tests/fhn.h:30-31 lists v before s; the TP06 rhs in
    # benchmarks/tentusscher_panfilov_2006_M_cell.py:13-33 puts Ca_i before
    # R_prime following dCa_i_dt/dR_prime_dt)
    m.states = OrderedDict((s, m.states[s]) for s in m.derivatives)
    m.source = text
    return m


def load_ode(path) -> ODEModel:
    """Load a ``.ode`` file (the ``.ode`` suffix may be omitted)."""
    p = Path(path)
    if not p.is_file() and p.suffix == "":
        p = p.with_suffix(".ode")
    if not p.is_file():
        raise FileNotFoundError(f"File {p} does not exist")
    name = p.stem.strip()
    return parse_ode_text(p.read_text(), name)
