"""Emit model source for every target from one :class:`ModelIR`.

Targets
-------
``emit_oracle_c``
    Plain C functions used by the CPU restatement in ``oracle/``.
``emit_goss_plugin``
    A ``goss::ParameterizedODE`` subclass plus ``extern "C" create_<Name>()``,
    the plugin shape of the reference generator (``python/goss/codegeneration.py:51-114``),
    so the reference's own compiled solvers can run the model.
``emit_device``
    CUDA ``__device__`` functions templated on the arithmetic type ``T``
    that the sm_100a solver kernels inline.

All three print the same :class:`Program` objects with the same printer, so
their arithmetic is identical operation for operation.
"""
from __future__ import annotations

import json
import re
from typing import Dict, List, Sequence, Tuple

import sympy as sp

from .ir import CONST, FIELD, STATE, TIME_CLS, Assign, ModelIR, Output, Program, count_ops
from .odeparse import TIME
from .ad import ReverseProgram
from .factor import factor_common
from .hoist import ConstantFolder
from .printer import CPrinter, c_double
from .sparse import LUStructure

_RESERVED = {
    "auto", "break", "case", "char", "const", "continue", "default", "do", "double", "else", "enum",
    "extern", "float", "for", "goto", "if", "inline", "int", "long", "register", "restrict", "return",
    "short", "signed", "sizeof", "static", "struct", "switch", "typedef", "union", "unsigned", "void",
    "volatile", "while", "bool", "class", "new", "delete", "this", "template", "typename", "namespace",
    "operator", "private", "public", "protected", "virtual", "friend", "true", "false", "time",
    "values", "states", "linear", "rhs", "monitored", "only_linear", "jac", "exp", "log", "sqrt", "pow",
    "floor", "ceil", "fabs", "abs", "sin", "cos", "tan", "tanh", "fmax", "fmin", "std", "goss",
}


def cxx_name(name: str) -> str:
    """Member/local name for the goss C++ class (gotran keeps plain names)."""
    return name + "_" if name in _RESERVED else name


def model_class_name(model_name: str) -> str:
    # gotran capitalises the ODE name (codegeneration.py:297)
    return model_name.capitalize()


def c_ident(model_name: str) -> str:
    s = re.sub(r"[^0-9A-Za-z_]", "_", model_name)
    if s[0].isdigit():
        s = "m_" + s
    return s


# ---------------------------------------------------------------------------
# helpers shared by the C-like targets
# ---------------------------------------------------------------------------

def _body_lines(prog: Program, pr_for, decl_for, out_for, split_code: List[str] = None) -> List[str]:
    lines: List[str] = []
    for idx, b in enumerate(prog.body):
        if prog.split is not None and idx == prog.split and split_code:
            lines.extend(split_code)
        if isinstance(b, Assign):
            lines.append(f"{decl_for(b)} = {pr_for(b.cls)(b.expr)};")
        else:
            lines.append(f"{out_for(b)} = {pr_for(STATE)(b.expr)};")
    if prog.split is not None and prog.split == len(prog.body) and split_code:
        lines.extend(split_code)
    return lines


class ModelSource:
    """Bundle of everything generated for one model + field-parameter set."""

    def __init__(self, ir: ModelIR, name: str = None, jacobian: bool = False):
        self.ir = ir
        self.model = ir.model
        self.name = name or self.model.name
        self.ident = c_ident(self.name)
        self.rhs = ir.rhs_program()
        self.lin = ir.linearized_program(split=True)
        self.linear_terms = ir.linear_terms()
        self.mon = ir.monitored_program() if ir.monitored else None
        # analytic Jacobian (the reference's code_params["generate_jacobian"])
        self.jac = ir.jacobian_program() if jacobian else None
        self.lus = LUStructure(ir.jacobian_structure())
        self.params = list(self.model.parameters)
        self.states = list(self.model.states)
        self.pindex = {p: i for i, p in enumerate(self.params)}
        self.sindex = {s: i for i, s in enumerate(self.states)}
        self.fparams = list(ir.field_parameters)
        self.findex = {p: i for i, p in enumerate(self.fparams)}
        self.inter_names = set(self.model.intermediates)

    # -- metadata -----------------------------------------------------------
    def metadata(self) -> Dict:
        return dict(
            name=self.name,
            ident=self.ident,
            class_name=model_class_name(self.name),
            state_names=self.states,
            parameter_names=self.params,
            initial_conditions=[float(v) for v in self.model.states.values()],
            default_parameters=[float(v) for v in self.model.parameters.values()],
            field_parameter_names=self.fparams,
            field_parameter_indices=[self.pindex[p] for p in self.fparams],
            field_state_names=list(self.ir.field_states),
            field_state_indices=[self.sindex[s] for s in self.ir.field_states],
            monitored_names=list(self.ir.monitored),
            linear_terms=self.linear_terms,
            intermediate_names=list(self.model.intermediates),
            op_census=dict(rhs=count_ops(self.rhs), linearized=count_ops(self.ir.linearized_program(split=False)),
                           linearized_split=self._split_census(),
                           **({"jacobian": count_ops(self.jac)} if self.jac is not None else {})),
            jacobian=self.jac is not None,
            jacobian_structure=[[int(v) for v in row] for row in self.lus.jac],
            lu_nnz=self.lus.nnz,
        )

    def _split_census(self) -> Dict[str, int]:
        """Per-evaluation census of the linearised program as the kernels run
        it: parameter-only sub-expressions folded into derived constants and
        every distinct exp/log/sqrt/reciprocal counted once (the elementary
        split of codegen/ad.py), time-only statements excluded."""
        folded = self._fold(self.ir.linearized_program(split=False))
        inter = {n: self.model.sym(n) for n in self.model.intermediates}
        rp = ReverseProgram(folded, [self.model.sym(s) for s in self.states],
                            [self.model.sym(p) for p in self.fparams], inter, reverse=False)
        body = [b for b in rp.forward if b.cls != TIME_CLS] + list(rp.outputs)
        return count_ops(Program("linearized_split", body, None))

    # =======================================================================
    # C restatement (oracle)
    # =======================================================================
    def _c_printer(self) -> CPrinter:
        def sym(s):
            n = s.name
            if s == TIME:
                return "time"
            if n in self.sindex:
                return f"s_{n}"
            if n in self.pindex:
                return f"p_{n}"
            return f"v_{n}"
        return CPrinter(sym)

    def _c_head(self) -> List[str]:
        lines = [f"const double s_{s} = states[{i}];" for i, s in enumerate(self.states)]
        lines += [f"const double p_{p} = params[{i}];" for i, p in enumerate(self.params)]
        return lines

    def emit_oracle_c(self) -> str:
        pr = self._c_printer()
        decl = lambda b: f"const double v_{b.name}"
        out = lambda b: f"{b.array}[{b.index}]"
        m = self.ident
        L = []
        L.append(f"/* Generated by goss_b200.codegen from the '{self.name}' model; do not edit. */")
        L.append("/* Test infrastructure: C restatement of the model consumed by the oracle. */")
        L.append("#include <math.h>")
        L.append('#include "goss_oracle.h"')
        L.append("")
        L.append("#if defined(__GNUC__)")
        L.append('#pragma GCC diagnostic ignored "-Wunused-variable"')
        L.append('#pragma GCC diagnostic ignored "-Wunused-parameter"')
        L.append("#endif")
        L.append("")
        L.append(f"static void {m}_rhs(const double* states, double time, const double* params, double* values)")
        L.append("{")
        L += ["  " + x for x in self._c_head()]
        L += ["  " + x for x in _body_lines(self.rhs, lambda c: pr, decl, out)]
        L.append("}")
        L.append("")
        L.append(f"static void {m}_linearized(const double* states, double time, const double* params,")
        L.append("    double* linear, double* rhs, int only_linear)")
        L.append("{")
        L += ["  " + x for x in self._c_head()]
        L += ["  " + x for x in _body_lines(self.lin, lambda c: pr, decl, out,
                                             split_code=["if (only_linear) return;"])]
        L.append("}")
        L.append("")
        if self.jac is not None:
            L.append(f"static void {m}_jacobian(const double* states, double time, const double* params, double* jac)")
            L.append("{")
            L += ["  " + x for x in self._c_head()]
            L += ["  " + x for x in _body_lines(self.jac, lambda c: pr, decl, out)]
            L.append("}")
            L.append("")
        if self.mon is not None:
            L.append(f"static void {m}_monitored(const double* states, double time, const double* params, double* monitored)")
            L.append("{")
            L += ["  " + x for x in self._c_head()]
            L += ["  " + x for x in _body_lines(self.mon, lambda c: pr, decl, out)]
            L.append("}")
            L.append("")
        ns, npar = len(self.states), len(self.params)
        L.append(f"static const double {m}_ic[{ns}] = {{" + ", ".join(c_double(v) for v in self.model.states.values()) + "};")
        L.append(f"static const double {m}_defaults[{npar}] = {{" + ", ".join(c_double(v) for v in self.model.parameters.values()) + "};" if npar else f"static const double {m}_defaults[1] = {{0.0}};")
        lt = self.linear_terms
        L.append(f"static const unsigned char {m}_linear_terms[{ns}] = {{" + ", ".join(str(v) for v in lt) + "};")
        nfp = len(self.fparams)
        fidx = [self.pindex[p] for p in self.fparams] or [0]
        L.append(f"static const unsigned {m}_field_param_index[{max(nfp,1)}] = {{" + ", ".join(str(v) for v in fidx) + "};")
        L.append("")
        L.append(f"const oracle_model* oracle_model_{m}(void)")
        L.append("{")
        L.append("  static oracle_model model;")
        L.append(f"  model.name = \"{self.name}\";")
        L.append(f"  model.num_states = {ns};")
        L.append(f"  model.num_params = {npar};")
        L.append(f"  model.num_field_params = {nfp};")
        L.append(f"  model.field_param_index = {m}_field_param_index;")
        L.append(f"  model.rhs = {m}_rhs;")
        L.append(f"  model.linearized = {m}_linearized;")
        L.append(f"  model.ic = {m}_ic;")
        L.append(f"  model.default_params = {m}_defaults;")
        L.append(f"  model.linear_terms = {m}_linear_terms;")
        L.append(f"  model.jacobian = {m + '_jacobian' if self.jac is not None else '0'};")
        L.append("  return &model;")
        L.append("}")
        return "\n".join(L) + "\n"

    # =======================================================================
    # goss C++ plugin (runs inside the reference's compiled solvers)
    # =======================================================================
    def emit_goss_plugin(self) -> str:
        cls = model_class_name(self.name)
        def sym(s):
            if s == TIME:
                return "time"
            return cxx_name(s.name)
        pr = CPrinter(sym, fn=dict(exp="std::exp", log="std::log", sqrt="std::sqrt", fabs="std::fabs",
                                   floor="std::floor", ceil="std::ceil", pow="std::pow", fmax="std::fmax",
                                   fmin="std::fmin", sin="std::sin", cos="std::cos", tan="std::tan",
                                   tanh="std::tanh"))
        decl = lambda b: f"const double {cxx_name(b.name)}"
        out = lambda b: f"{b.array}[{b.index}]"
        head = [f"const double {cxx_name(s)} = states[{i}];" for i, s in enumerate(self.states)]
        ns, npar = len(self.states), len(self.params)
        nfs, nfp, nmon = len(self.ir.field_states), len(self.fparams), len(self.ir.monitored)
        I = lambda n: " " * n
        L = []
        guard = self.ident.upper() + "_GOSS_PLUGIN_H"
        L.append(f"// Generated by goss_b200.codegen from the '{self.name}' model; do not edit.")
        L.append("// goss::ParameterizedODE plugin consumed by the oracle build of the reference solvers.")
        L.append(f"#ifndef {guard}")
        L.append(f"#define {guard}")
        L.append("#include <cmath>")
        L.append("#include <memory>")
        L.append("#include <stdexcept>")
        L.append('#include "goss/ParameterizedODE.h"')
        L.append("")
        L.append("namespace goss {")
        L.append(f"class {cls} : public ParameterizedODE")
        L.append("{")
        L.append("  public:")
        init = ", ".join(f"{cxx_name(p)}({c_double(v)})" for p, v in self.model.parameters.items())
        L.append(f"    {cls}() : ParameterizedODE({ns}, {npar}, {nfs}, {nfp}, {nmon})" + (f", {init}" if init else ""))
        L.append("    {")
        for i, s in enumerate(self.states):
            L.append(f'        _state_names[{i}] = "{s}";')
        for i, p in enumerate(self.params):
            L.append(f'        _parameter_names[{i}] = "{p}";')
        for i, s in enumerate(self.ir.field_states):
            L.append(f'        _field_state_names[{i}] = "{s}";')
            L.append(f"        _field_state_indices[{i}] = {self.sindex[s]};")
        for i, p in enumerate(self.fparams):
            L.append(f'        _field_parameter_names[{i}] = "{p}";')
        for i, mname in enumerate(self.ir.monitored):
            L.append(f'        _monitored_names[{i}] = "{mname}";')
        for p in self.params:
            L.append(f'        _param_to_value["{p}"] = &{cxx_name(p)};')
        for i, f in enumerate(self.linear_terms):
            if f:
                L.append(f"        _linear_terms[{i}] = 1;")
        L.append("    }")
        cinit = ", ".join(f"{cxx_name(p)}(ode.{cxx_name(p)})" for p in self.params)
        L.append(f"    {cls}(const {cls}& ode) : ParameterizedODE(ode)" + (f", {cinit}" if cinit else "") + " {}")
        L.append("")
        L.append("    void eval(const double* states, double time, double* values)")
        L.append("    {")
        L += [I(8) + x for x in head + _body_lines(self.rhs, lambda c: pr, decl, out)]
        L.append("    }")
        L.append("")
        L.append("    void linearized_eval(const double* states, double time, double* linear, double* rhs,")
        L.append("                         bool only_linear) const")
        L.append("    {")
        L += [I(8) + x for x in head + _body_lines(self.lin, lambda c: pr, decl, out,
                                                  split_code=["if (only_linear) return;"])]
        L.append("    }")
        L.append("")
        if self.jac is not None:
            L.append("    // Compute analytic jacobian")
            L.append("    void compute_jacobian(double* states, double time, double* jac)")
            L.append("    {")
            L += [I(8) + x for x in head + _body_lines(self.jac, lambda c: pr, decl, out)]
            L.append("    }")
            L.append("")
        L.append("    void get_ic(goss::DoubleVector* values) const")
        L.append("    {")
        L.append("        values->n = _num_states;")
        L.append("        values->data.reset(new double[_num_states]);")
        for i, v in enumerate(self.model.states.values()):
            L.append(f"        values->data[{i}] = {c_double(v)};")
        L.append("    }")
        L.append("")
        L.append("    std::shared_ptr<ODE> copy() const { return std::make_shared<" + cls + ">(*this); }")
        L.append("")
        L.append("    void eval_monitored(const double* states, double time, double* monitored) const")
        L.append("    {")
        if self.mon is None:
            L.append(f'        throw std::runtime_error("No monitored in the \\\'{cls}\\\' model.");')
        else:
            L += [I(8) + x for x in head + _body_lines(self.mon, lambda c: pr, decl, out)]
        L.append("    }")
        L.append("")
        L.append("    void set_field_parameters(const double* field_params)")
        L.append("    {")
        for i, p in enumerate(self.fparams):
            L.append(f"        {cxx_name(p)} = field_params[{i}];")
        if not self.fparams:
            L.append("        (void)field_params;")
        L.append("    }")
        L.append("")
        L.append("  private:")
        if self.params:
            L.append("    double " + ", ".join(cxx_name(p) for p in self.params) + ";")
        L.append("};")
        L.append("}  // namespace goss")
        L.append("")
        L.append(f'extern "C" __attribute__((visibility("default"))) goss::ParameterizedODE* create_{cls}()')
        L.append("{")
        L.append(f"    return new goss::{cls};")
        L.append("}")
        L.append("#endif")
        return "\n".join(L) + "\n"

    # =======================================================================
    # CUDA device code
    # =======================================================================
    def _dev_printers(self, split: bool = False):
        """Printers for arithmetic type T and for double (time-only) context;
        ``split``: the T printer of the split forms, whose exponentials with a
        numeric coefficient go through exp2 (one multiply fewer)."""
        def make(ctx_double: bool):
            def sym(s):
                n = s.name
                if s == TIME:
                    return "time" if ctx_double else "T(time)"
                if n in self.sindex:
                    return f"s_{n}"
                if n in self.pindex:
                    if n in self.findex:
                        j = self.findex[n]
                        return f"double(F[{j}])" if ctx_double else f"F[{j}]"
                    k = self.pindex[n]
                    return f"PD[{k}]" if ctx_double else f"P[{k}]"
                if n.startswith("__seed_linear_"):
                    return f"abar[{int(n[len('__seed_linear_'):])}]"
                if n.startswith("__seed_rhs_"):
                    return f"bbar[{int(n[len('__seed_rhs_'):])}]"
                if n.startswith("__seed_values_"):
                    return f"bbar[{int(n[len('__seed_values_'):])}]"
                if n.startswith("__adj_"):
                    return f"a_{n[len('__adj_'):]}"
                if n.startswith("__c"):
                    # derived constant, stored after the parameters
                    k = len(self.params) + int(n[3:])
                    return f"PD[{k}]" if ctx_double else f"P[{k}]"
                # intermediate: its declared type follows its class
                cls = self._cls_of(n)
                if cls == TIME_CLS and not ctx_double:
                    return f"T(v_{n})"
                return f"v_{n}"
            if ctx_double:
                fn = dict(exp="exp", log="log", sqrt="sqrt", fabs="fabs", floor="floor", ceil="ceil",
                          pow="pow", fmax="fmax", fmin="fmin")
                lit = c_double
            else:
                fn = dict(exp="gexp", exp2="gexp2", log="glog", sqrt="gsqrt", fabs="gfabs", floor="gfloor",
                          ceil="gceil", pow="gpow", fmax="gfmax", fmin="gfmin", sin="gsin", cos="gcos", tan="gtan",
                          tanh="gtanh")
                lit = lambda v: f"T({c_double(v)})"
            return CPrinter(sym, fn=fn, lit=lit, exp2_fold=split and not ctx_double)
        return make(False), make(True)

    def _programs(self) -> Tuple[Program, ...]:
        return (self.rhs, self.lin) + ((self.mon,) if self.mon else ()) + ((self.jac,) if self.jac else ())

    def _cls_of(self, name: str) -> int:
        return self._cls_map.get(name, STATE)

    @property
    def _cls_map(self) -> Dict[str, int]:
        if not hasattr(self, "_cls_cache"):
            d = {}
            for prog in self._programs():
                for b in prog.assigns():
                    d[b.name] = b.cls
            self._cls_cache = d
        return self._cls_cache

    def _dev_body(self, prog: Program) -> List[str]:
        prT, prD = self._dev_printers()
        def pr_for(cls):
            return prD if cls == TIME_CLS else prT
        def decl(b):
            t = "double" if b.cls == TIME_CLS else "T"
            return f"const {t} v_{b.name}"
        out = lambda b: f"{b.array}[{b.index}]"
        p2 = Program(prog.name, self._fold(prog).body, None)
        return _body_lines(p2, pr_for, decl, out)

    # -- parameter-only sub-expressions become derived constants ----------------
    @property
    def folder(self) -> ConstantFolder:
        if not hasattr(self, "_folder"):
            uniform = {self.model.sym(p) for p in self.params if p not in self.findex}
            const_inter = {}
            for prog in self._programs():
                for b in prog.assigns():
                    if b.cls == CONST:
                        const_inter[self.model.sym(b.name)] = b.expr
            self._folder = ConstantFolder(uniform, const_inter)
            self._const_inter = const_inter
        return self._folder

    def _fold(self, prog: Program) -> Program:
        f = self.folder
        body = []
        for b in prog.body:
            if isinstance(b, Assign):
                if b.cls == CONST:
                    continue
                body.append(Assign(b.name, f(b.expr), b.cls))
            else:
                body.append(Output(b.array, b.index, f(b.expr)))
        return Program(prog.name, body, None)

    def _dev_vjp_lines(self, prog: Program, arrays: Dict[str, Tuple[str, str]], seed_call: str) -> List[str]:
        """Body of a VJP: forward sweep, the caller's seed, the reverse sweep.

        arrays maps each output array of ``prog`` to (value array, cotangent
        array) names; ``seed_call`` hands both to the caller's seed."""
        folded = self._fold(prog)
        inter = {n: self.model.sym(n) for n in self.model.intermediates}
        rp = ReverseProgram(folded, [self.model.sym(s) for s in self.states],
                            [self.model.sym(p) for p in self.fparams], inter)
        prT, prD = self._dev_printers(split=True)
        lines = []
        for b in rp.forward:
            if b.cls == TIME_CLS:
                lines.append(f"const double v_{b.name} = {prD(b.expr)};")
            else:
                lines.append(f"const T v_{b.name} = {prT(factor_common(b.expr))};")
        # the values themselves, then the caller's cotangents for them
        n = len(self.states)
        decl = ", ".join(f"{v}[{n}], {c}[{n}]" for v, c in arrays.values())
        lines.append(f"T {decl};")
        for o in rp.outputs:
            lines.append(f"{arrays[o.array][0]}[{o.index}] = {prT(factor_common(o.expr))};")
        for arr, (val, _) in arrays.items():
            for i in range(n):
                if not any(o.array == arr and o.index == i for o in rp.outputs):
                    lines.append(f"{val}[{i}] = T(0.0);")
        lines.append(seed_call)
        for adj, e in rp.reverse:
            lines.append(f"const T a_{adj.name[len('__adj_'):]} = {prT(factor_common(e))};")
        for i, e in enumerate(rp.state_bar):
            lines.append(f"ybar[{i}] = {prT(factor_common(e)) if e != 0 else 'T(0.0)'};")
        for k, e in enumerate(rp.field_bar):
            lines.append(f"Fbar[{k}] = {prT(factor_common(e)) if e != 0 else 'T(0.0)'};")
        return lines

    def _packed_jacobian(self) -> Program:
        """The analytic Jacobian program with its outputs at the packed
        positions of the LU structure (entries outside it are exactly 0)."""
        n = len(self.states)
        body = []
        for b in self.jac.body:
            if isinstance(b, Output):
                r, c = divmod(b.index, n)
                if self.lus.nz(r, c):
                    body.append(Output("jac", self.lus.pos[(r, c)], b.expr))
                elif b.expr != 0:
                    raise AssertionError(f"jac[{r}][{c}] outside the dependency structure")
            else:
                body.append(b)
        return Program("jacobian_packed", body, None)

    def _dev_split_lines(self, prog: Program, arrays: Dict[str, str], size: int = None) -> List[str]:
        """Body of ``prog`` with every distinct exp/log/sqrt/pow/reciprocal of
        state-dependent operands computed once (the elementary split of
        codegen/ad.py) and common factors pulled out of sums (codegen/factor.py);
        ``arrays`` names the output array of each of its output arrays, each of
        ``size`` entries (default: the number of states)."""
        folded = self._fold(prog)
        inter = {n: self.model.sym(n) for n in self.model.intermediates}
        rp = ReverseProgram(folded, [self.model.sym(s) for s in self.states],
                            [self.model.sym(p) for p in self.fparams], inter, reverse=False)
        prT, prD = self._dev_printers(split=True)
        lines = []
        for b in rp.forward:
            if b.cls == TIME_CLS:
                lines.append(f"const double v_{b.name} = {prD(b.expr)};")
            else:
                lines.append(f"const T v_{b.name} = {prT(factor_common(b.expr))};")
        n = len(self.states) if size is None else size
        for o in rp.outputs:
            lines.append(f"{arrays[o.array]}[{o.index}] = {prT(factor_common(o.expr))};")
        for arr, name in arrays.items():
            for i in range(n):
                if not any(o.array == arr and o.index == i for o in rp.outputs):
                    lines.append(f"{name}[{i}] = T(0.0);")
        return lines

    def _t0_lines(self, binds, outs, prT, prD) -> List[str]:
        """f0 = f(y, t0) next to f1 = f(y, time) written just before: only the
        statements that depend on the time (the stimulus and what it feeds) are
        evaluated again at t0; every other row of f0 is the row of f1."""
        import sympy

        n = len(self.states)
        syms = {}
        for e in [b.expr for b in binds] + [o.expr for o in outs.values()]:
            for sym in e.free_symbols:
                syms.setdefault(sym.name, sym)
        t0 = sympy.Symbol("__tzero")
        sub, cone = {TIME: t0}, set()
        lines = ["const double v___tzero = t0;"]
        for b in binds:
            names = {x.name for x in b.expr.free_symbols}
            if b.cls == TIME_CLS or TIME in b.expr.free_symbols or names & cone:
                cone.add(b.name)
                new = sympy.Symbol(f"{b.name}__tz")
                e = b.expr.xreplace(sub)
                if b.cls == TIME_CLS:
                    lines.append(f"const double v_{new.name} = {prD(e)};")
                else:
                    lines.append(f"const T v_{new.name} = {prT(factor_common(e))};")
                sub[syms.get(b.name, sympy.Symbol(b.name))] = new
        for r in range(n):
            o = outs.get(r)
            if o is None:
                lines.append(f"f0[{r}] = T(0.0);")
            elif TIME in o.expr.free_symbols or {x.name for x in o.expr.free_symbols} & cone:
                lines.append(f"f0[{r}] = {prT(factor_common(o.expr.xreplace(sub)))};")
            else:
                lines.append(f"f0[{r}] = f1[{r}];")
        return lines

    def _dev_rhs_jacobian_lines(self, with_t0: bool = False) -> List[str]:
        """Body of ``rhs_jacobian``: f(y) (``rhs_split``'s outputs) and the
        analytic Jacobian into the packed Newton matrix from one split program,
        so their exponentials, reciprocals and intermediates are computed once."""
        rhs, jac = self.rhs, self._packed_jacobian()
        names = {b.name for b in rhs.body if isinstance(b, Assign)}
        body = [b for b in rhs.body if isinstance(b, Assign)]
        body += [b for b in jac.body if isinstance(b, Assign) and b.name not in names]
        body += [b for b in rhs.body if isinstance(b, Output)] + [b for b in jac.body if isinstance(b, Output)]
        folded = self._fold(Program("rhs_jacobian", body, None))
        inter = {n: self.model.sym(n) for n in self.model.intermediates}
        rp = ReverseProgram(folded, [self.model.sym(s) for s in self.states],
                            [self.model.sym(p) for p in self.fparams], inter, reverse=False)
        prT, prD = self._dev_printers(split=True)
        lines = []
        for b in rp.forward:
            if b.cls == TIME_CLS:
                lines.append(f"const double v_{b.name} = {prD(b.expr)};")
            else:
                lines.append(f"const T v_{b.name} = {prT(factor_common(b.expr))};")
        arrays, sizes = {"values": "f1", "jac": "J"}, {"values": len(self.states), "jac": self.lus.nnz}
        for o in rp.outputs:
            lines.append(f"{arrays[o.array]}[{o.index}] = {prT(factor_common(o.expr))};")
        for arr, name in arrays.items():
            done = {o.index for o in rp.outputs if o.array == arr}
            lines += [f"{name}[{i}] = T(0.0);" for i in range(sizes[arr]) if i not in done]
        if with_t0:
            lines += self._t0_lines(list(rp.forward), {o.index: o for o in rp.outputs if o.array == "values"},
                                    prT, prD)
        return lines

    def _dev_rhs_jacobian_sel_lines(self) -> List[str]:
        """Body of ``rhs_jacobian_sel``: ``rhs2_jacobian``'s program with the
        statements that only the Jacobian needs, and the Jacobian's outputs,
        under ``if (want_jac)``, and f0's time-dependent statements under
        ``if (want_f0)``: one inlined copy of the model serves every Newton
        iteration (f alone, f and the Jacobian, f at two times)."""
        rhs, jac = self.rhs, self._packed_jacobian()
        names = {b.name for b in rhs.body if isinstance(b, Assign)}
        body = [b for b in rhs.body if isinstance(b, Assign)]
        body += [b for b in jac.body if isinstance(b, Assign) and b.name not in names]
        body += [b for b in rhs.body if isinstance(b, Output)] + [b for b in jac.body if isinstance(b, Output)]
        folded = self._fold(Program("rhs_jacobian", body, None))
        inter = {n: self.model.sym(n) for n in self.model.intermediates}
        rp = ReverseProgram(folded, [self.model.sym(s) for s in self.states],
                            [self.model.sym(p) for p in self.fparams], inter, reverse=False)
        prT, prD = self._dev_printers(split=True)
        fwd = list(rp.forward)
        f_outs = [o for o in rp.outputs if o.array == "values"]
        j_outs = [o for o in rp.outputs if o.array == "jac"]
        by_name = {b.name: b for b in fwd}
        need, stack = set(), [x.name for o in f_outs for x in o.expr.free_symbols]
        while stack:
            nm = stack.pop()
            if nm in by_name and nm not in need:
                need.add(nm)
                stack.extend(x.name for x in by_name[nm].expr.free_symbols)

        def stmt(b):
            if b.cls == TIME_CLS:
                return f"const double v_{b.name} = {prD(b.expr)};"
            return f"const T v_{b.name} = {prT(factor_common(b.expr))};"

        n = len(self.states)
        lines = [stmt(b) for b in fwd if b.name in need]
        lines += [f"f1[{o.index}] = {prT(factor_common(o.expr))};" for o in f_outs]
        done = {o.index for o in f_outs}
        lines += [f"f1[{i}] = T(0.0);" for i in range(n) if i not in done]
        lines.append("if (want_jac) {")
        lines += ["  " + stmt(b) for b in fwd if b.name not in need]
        lines += [f"  J[{o.index}] = {prT(factor_common(o.expr))};" for o in j_outs]
        done = {o.index for o in j_outs}
        lines += [f"  J[{i}] = T(0.0);" for i in range(self.lus.nnz) if i not in done]
        lines.append("}")
        lines.append("if (want_f0) {")
        lines += ["  " + x for x in self._t0_lines([b for b in fwd if b.name in need],
                                                  {o.index: o for o in f_outs}, prT, prD)]
        lines.append("}")
        return lines

    def _dev_fd_jacobian_lines(self, with_rhs: bool = False, with_t0: bool = False,
                               select: bool = False) -> List[str]:
        """Body of ``fd_jacobian``: the forward-difference Jacobian of the split
        right-hand side into the packed Newton matrix.  The unperturbed
        statements are evaluated once; column i then recomputes, for
        y + delta_i e_i, only the statements of its structural rows that depend
        on state i (the others keep their unperturbed values, which is what
        re-evaluating them would give), and stores (f2 - f1) / delta_i at those
        rows.  delta_i = sqrt(1e-15 max(1e-5, |y_i|)) as in ODE::compute_jacobian."""
        import sympy

        folded = self._fold(self.rhs)
        inter = {n: self.model.sym(n) for n in self.model.intermediates}
        rp = ReverseProgram(folded, [self.model.sym(s) for s in self.states],
                            [self.model.sym(p) for p in self.fparams], inter, reverse=False)
        prT, prD = self._dev_printers(split=True)
        binds = list(rp.forward)
        bmap = {b.name: b for b in binds}
        outs = {o.index: o for o in rp.outputs if o.array == "values"}
        n = len(self.states)
        syms = {}
        for e in [b.expr for b in binds] + [o.expr for o in outs.values()]:
            for sym in e.free_symbols:
                syms.setdefault(sym.name, sym)
        sidx = {self.model.sym(st).name: i for i, st in enumerate(self.states)}
        deps = {}  # binding -> states it depends on, transitively
        for b in binds:
            d = set()
            for sym in b.expr.free_symbols:
                if sym.name in sidx:
                    d.add(sidx[sym.name])
                elif sym.name in deps:
                    d |= deps[sym.name]
            deps[b.name] = d
        lines = []
        for b in binds:
            if b.cls == TIME_CLS:
                lines.append(f"const double v_{b.name} = {prD(b.expr)};")
            else:
                lines.append(f"const T v_{b.name} = {prT(factor_common(b.expr))};")
        if with_rhs:  # f1 = f(y): the outputs of rhs_split, from the same statements
            for r in range(n):
                lines.append(f"f1[{r}] = {prT(factor_common(outs[r].expr)) if r in outs else 'T(0.0)'};")
            if with_t0:
                lines += self._t0_lines(binds, outs, prT, prD)
        if select:  # the columns only if want_jac (J is left as it is otherwise)
            lines += ["if (want_jac) {", "fd_clear(J);"]
        for i in range(n):
            rows = [r for r in range(n) if self.lus.jac[r][i] and r in outs]
            if not rows:
                continue
            need, stack = set(), [sym.name for r in rows for sym in outs[r].expr.free_symbols]
            while stack:
                name = stack.pop()
                if name in bmap and name not in need:
                    need.add(name)
                    stack += [sym.name for sym in bmap[name].expr.free_symbols]
            state_sym = syms.get(self.model.sym(self.states[i]).name, self.model.sym(self.states[i]))
            sub = {state_sym: sympy.Symbol(f"__yp{i}")}
            lines.append("{")
            lines.append(f"  const double d = sqrt(1e-15 * (1e-5 > fabs(double(y[{i}])) ? 1e-5 : fabs(double(y[{i}]))));")
            lines.append(f"  const T v___yp{i} = T(double(y[{i}]) + d);")
            for b in binds:
                if b.name in need and i in deps[b.name]:
                    new = sympy.Symbol(f"{b.name}__k{i}")
                    lines.append(f"  const T v_{new.name} = {prT(factor_common(b.expr.xreplace(sub)))};")
                    sub[syms.get(b.name, sympy.Symbol(b.name))] = new
            for r in rows:
                f2 = prT(factor_common(outs[r].expr.xreplace(sub)))
                lines.append(f"  J[{self.lus.pos[(r, i)]}] = (({f2}) - f1[{r}]) / d;")
            lines.append("}")
        if select:
            lines.append("}")
        return lines

    def _derived_host_lines(self) -> List[str]:
        """Host code filling C[k] with the derived constants from P."""
        def sym(s):
            n = s.name
            if n in self.pindex:
                return f"P[{self.pindex[n]}]"
            return f"v_{n}"
        pr = CPrinter(sym)
        lines = []
        order = [b for prog in self._programs() for b in prog.assigns() if b.cls == CONST]
        seen = set()
        for b in order:
            if b.name in seen:
                continue
            seen.add(b.name)
            lines.append(f"const double v_{b.name} = {pr(b.expr)};")
        for k, (s, e) in enumerate(self.folder.derived):
            lines.append(f"C[{k}] = {pr(e)};")
        if not seen:
            pass
        return lines

    def emit_device(self, struct_name: str = None) -> str:
        # one struct per variant, so several variants can share a translation unit
        cls = struct_name or model_class_name(self.name)
        ns, npar, nfp = len(self.states), len(self.params), len(self.fparams)
        L = []
        guard = cls.upper() + "_DEVICE_CUH"
        L.append(f"// Generated by goss_b200.codegen from the '{self.name}' model; do not edit.")
        L.append("// Device-side model: rhs and linearised rhs templated on the arithmetic type T.")
        L.append(f"#ifndef {guard}")
        L.append(f"#define {guard}")
        L.append('#include "goss_device_math.cuh"')
        L.append("")
        L.append("namespace goss_b200 { namespace models {")
        L.append("")
        L.append(f"struct {cls} {{")
        L.append(f'  static constexpr const char* name = "{self.name}";')
        L.append(f"  static constexpr int num_states = {ns};")
        L.append(f"  static constexpr int num_params = {npar};")
        L.append(f"  static constexpr int num_field_params = {nfp};")
        L.append(f"  static constexpr int num_monitored = {len(self.ir.monitored)};")
        L.append("")
        head = [f"const T s_{s} = y[{i}];" for i, s in enumerate(self.states)]
        sig = ("const T* __restrict__ y, const double time, const T* __restrict__ P, "
               "const double* __restrict__ PD, const T* __restrict__ F")
        L.append("  // values = f(y, time)")
        L.append("  template <typename T>")
        L.append(f"  __device__ static __forceinline__ void rhs({sig}, T* __restrict__ values)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_body(self.rhs)]
        L.append("    (void)time; (void)P; (void)PD; (void)F;")
        L.append("  }")
        L.append("")
        lin_full = self.ir.linearized_program(split=False)
        rhs_lines = self._dev_body(self.rhs)
        lin_lines = self._dev_body(lin_full)
        mon_lines = self._dev_body(self.mon) if self.mon is not None else []
        jac_lines = (self._dev_split_lines(self._packed_jacobian(), {"jac": "J"}, self.lus.nnz)
                     if self.jac is not None else [])
        nder = len(self.folder.derived)
        L.insert(L.index(f"  static constexpr int num_monitored = {len(self.ir.monitored)};") + 1,
                 f"  static constexpr int num_derived = {nder};")
        lin_idx = [i for i, f in enumerate(self.linear_terms) if f]
        cond = " || ".join(f"i == {i}" for i in lin_idx) or "false"
        L.insert(L.index(f"  static constexpr int num_derived = {nder};") + 1,
                 "  // the reference generator's linear-term flags (RL1/RL2 use the exponential update for these)\n"
                 f"  __host__ __device__ static constexpr bool linear_term(int i) {{ return {cond}; }}")
        L += self._dev_lu_lines(head, sig, jac_lines)
        L.append("  // derived constants: parameter-only sub-expressions, evaluated once per")
        L.append("  // launch on the host in FP64 and stored after the parameters")
        L.append("  static void derived(const double* P, double* C)")
        L.append("  {")
        L += ["    " + x for x in self._derived_host_lines()]
        L.append("    (void)P; (void)C;")
        L.append("  }")
        L.append("")
        L.append("  // rhs = f(y, time), linear[i] = d f_i / d y_i")
        L.append("  template <typename T>")
        L.append(f"  __device__ static __forceinline__ void linearized({sig}, T* __restrict__ linear, T* __restrict__ rhs)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_body(lin_full)]
        L.append("    (void)time; (void)P; (void)PD; (void)F;")
        L.append("  }")
        L.append("")
        L.append("  // linearized with every distinct transcendental and reciprocal of a state-dependent")
        L.append("  // operand evaluated once (the FP32 kernels' form; FP64 keeps the reference's operations)")
        L.append("  template <typename T>")
        L.append(f"  __device__ static __forceinline__ void linearized_split({sig}, T* __restrict__ linear, T* __restrict__ rhs)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_split_lines(lin_full, {"linear": "linear", "rhs": "rhs"})]
        L.append("    (void)time; (void)P; (void)PD; (void)F;")
        L.append("  }")
        L.append("")
        L.append("  // rhs in the same split form")
        L.append("  template <typename T>")
        L.append(f"  __device__ static __forceinline__ void rhs_split({sig}, T* __restrict__ values)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_split_lines(self.rhs, {"values": "values"})]
        L.append("    (void)time; (void)P; (void)PD; (void)F;")
        L.append("  }")
        L.append("")
        L.append("  // forward-difference Jacobian of rhs_split at y into the packed Newton matrix (structural")
        L.append("  // entries; fd_clear sets the others): f1 = f(y, time); column i recomputes only the")
        L.append("  // statements of its rows that depend on state i")
        L.append("  template <typename T, class A>")
        L.append(f"  __device__ static __forceinline__ void fd_jacobian({sig}, const T* __restrict__ f1, A J)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_fd_jacobian_lines()]
        L.append("    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;")
        L.append("  }")
        L.append("")
        if self.jac is not None:
            L.append("  // f1 = f(y, time) (rhs_split) and the analytic Jacobian into the packed Newton matrix,")
            L.append("  // sharing their exponentials, reciprocals and intermediates")
            L.append("  template <typename T, class A>")
            L.append(f"  __device__ static __forceinline__ void rhs_jacobian({sig}, T* __restrict__ f1, A J)")
            L.append("  {")
            L += ["    " + x for x in head + self._dev_rhs_jacobian_lines()]
            L.append("    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;")
            L.append("  }")
            L.append("")
            L.append("  // the same, also writing f0 = f(y, t0) (only the time-dependent statements again)")
            L.append("  template <typename T, class A>")
            L.append(f"  __device__ static __forceinline__ void rhs2_jacobian({sig}, const double t0,")
            L.append("      T* __restrict__ f0, T* __restrict__ f1, A J)")
            L.append("  {")
            L += ["    " + x for x in head + self._dev_rhs_jacobian_lines(with_t0=True)]
            L.append("    (void)time; (void)t0; (void)P; (void)PD; (void)F; (void)f0; (void)f1; (void)J;")
            L.append("  }")
            L.append("")
            L.append("  // f1 = f(y, time); the Jacobian only if want_jac (J is left as it is otherwise), f0 =")
            L.append("  // f(y, t0) only if want_f0: rhs2_jacobian with its parts selected at run time")
            L.append("  template <typename T, class A>")
            L.append(f"  __device__ static __forceinline__ void rhs_jacobian_sel({sig}, const double t0,")
            L.append("      const bool want_f0, const bool want_jac, T* __restrict__ f0, T* __restrict__ f1, A J)")
            L.append("  {")
            L += ["    " + x for x in head + self._dev_rhs_jacobian_sel_lines()]
            L.append("    (void)time; (void)t0; (void)P; (void)PD; (void)F; (void)f0; (void)f1; (void)J;")
            L.append("  }")
            L.append("")
        L.append("  // the same, also writing f1 = f(y, time) (rhs_split) from its unperturbed statements")
        L.append("  template <typename T, class A>")
        L.append(f"  __device__ static __forceinline__ void rhs_fd_jacobian({sig}, T* __restrict__ f1, A J)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_fd_jacobian_lines(with_rhs=True)]
        L.append("    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;")
        L.append("  }")
        L.append("")
        L.append("  // f1 = f(y, time), and the forward-difference Jacobian only if want_jac (J is left as it")
        L.append("  // is otherwise): rhs_fd_jacobian with its columns selected at run time")
        L.append("  template <typename T, class A>")
        L.append(f"  __device__ static __forceinline__ void rhs_fd_jacobian_sel({sig}, const bool want_jac,")
        L.append("      T* __restrict__ f1, A J)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_fd_jacobian_lines(with_rhs=True, select=True)]
        L.append("    (void)time; (void)P; (void)PD; (void)F; (void)f1; (void)J;")
        L.append("  }")
        L.append("")
        L.append("  // the same, also writing f0 = f(y, t0) (only the time-dependent statements again)")
        L.append("  template <typename T, class A>")
        L.append(f"  __device__ static __forceinline__ void rhs2_fd_jacobian({sig}, const double t0,")
        L.append("      T* __restrict__ f0, T* __restrict__ f1, A J)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_fd_jacobian_lines(with_rhs=True, with_t0=True)]
        L.append("    (void)time; (void)t0; (void)P; (void)PD; (void)F; (void)f0; (void)f1; (void)J;")
        L.append("  }")
        L.append("")
        L.append("  // vector-Jacobian product of linearized (reverse mode, generated): after the forward")
        L.append("  // sweep seed(linear, rhs, abar, bbar) supplies the cotangents of the outputs, then")
        L.append("  // ybar = abar^T d(linear)/dy + bbar^T d(rhs)/dy and Fbar likewise for the field parameters")
        L.append("  template <typename T, class Seed>")
        L.append(f"  __device__ static __forceinline__ void linearized_vjp({sig}, Seed&& seed,")
        L.append("      T* __restrict__ ybar, T* __restrict__ Fbar)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_vjp_lines(
            lin_full, {"linear": ("lin_v", "abar"), "rhs": ("rhs_v", "bbar")}, "seed(lin_v, rhs_v, abar, bbar);")]
        L.append("    (void)time; (void)P; (void)PD; (void)F; (void)abar; (void)bbar; (void)Fbar;")
        L.append("  }")
        L.append("")
        L.append("  // vector-Jacobian product of rhs (reverse mode, generated): after the forward sweep")
        L.append("  // seed(values, bbar) supplies the cotangents of the values, then ybar = bbar^T df/dy")
        L.append("  // and Fbar = bbar^T df/dF")
        L.append("  template <typename T, class Seed>")
        L.append(f"  __device__ static __forceinline__ void rhs_vjp({sig}, Seed&& seed,")
        L.append("      T* __restrict__ ybar, T* __restrict__ Fbar)")
        L.append("  {")
        L += ["    " + x for x in head + self._dev_vjp_lines(self.rhs, {"values": ("f_v", "bbar")},
                                                             "seed(f_v, bbar);")]
        L.append("    (void)time; (void)P; (void)PD; (void)F; (void)bbar; (void)Fbar;")
        L.append("  }")
        if self.mon is not None:
            L.append("")
            L.append("  template <typename T>")
            L.append(f"  __device__ static __forceinline__ void monitored_values({sig}, T* __restrict__ monitored)")
            L.append("  {")
            L += ["    " + x for x in head + self._dev_body(self.mon)]
            L.append("    (void)time; (void)P; (void)PD; (void)F;")
            L.append("  }")
        L.append("};")
        L.append("")
        L.append("}}  // namespace goss_b200::models")
        L.append("#endif")
        return "\n".join(L) + "\n"

    def _dev_lu_lines(self, head: List[str], sig: str, jac_lines: List[str]) -> List[str]:
        """Packed Newton matrix of the implicit solvers: the LU structure of
        I - h*alpha*J, the structure-aware factorisation and solve
        (codegen/sparse.py), the forward-difference column store and, with the
        analytic Jacobian, its evaluation into the packed layout."""
        lus, n = self.lus, len(self.states)
        I4 = lambda lines: ["    " + x for x in lines]
        L = []
        L.append(f"  // Newton matrix: {lus.nnz} packed entries (the Jacobian's {sum(map(sum, lus.jac))} structural")
        L.append("  // non-zeros, the diagonal and the LU fill-in; row-major over the structure)")
        L.append(f"  static constexpr int lu_nnz = {lus.nnz};")
        L.append(f"  static constexpr bool has_jacobian = {'true' if self.jac is not None else 'false'};")
        L.append("  // J := scale*J + I")
        L.append("  template <class A>")
        L.append("  __device__ static __forceinline__ void lu_shift(A J, const double scale)")
        L.append("  {")
        L += I4(lus.shift_lines("J", "scale"))
        L.append("  }")
        L.append("  // D := scale*S + I")
        L.append("  template <class A, class B>")
        L.append("  __device__ static __forceinline__ void lu_copy_shift(A S, B D, const double scale)")
        L.append("  {")
        L += I4(lus.copy_shift_lines("S", "D", "scale"))
        L.append("  }")
        L.append("  // in-place Doolittle LU without pivoting over the structure")
        L.append("  template <class A>")
        L.append("  __device__ static __forceinline__ void lu_factorize(A J)")
        L.append("  {")
        L += I4(lus.lu_factorize_lines("J"))
        L.append("  }")
        L.append("  // x = (LU)^-1 b, forward then backward substitution; b and x may alias")
        L.append("  template <class A>")
        L.append("  __device__ static __forceinline__ void lu_solve(A J, const double* b, double* x)")
        L.append("  {")
        L += I4(lus.solve_lines("J", "b", "x"))
        L.append("  }")
        L.append("  // forward differences: zero the entries outside the Jacobian's structure, then")
        L.append("  // column i = (f2 - f1) / delta at its structural rows")
        L.append("  template <class A>")
        L.append("  __device__ static __forceinline__ void fd_clear(A J)")
        L.append("  {")
        L += I4(lus.clear_extra_lines("J"))
        L.append("    (void)J;")
        L.append("  }")
        L.append("  template <class A>")
        L.append("  __device__ static __forceinline__ void fd_column(const int i, const double* f1, const double* f2,")
        L.append("                                                   const double delta, A J)")
        L.append("  {")
        L += I4(lus.fd_column_lines("J"))
        L.append("  }")
        L.append("  // dense row-major copy: out(r*n + c, value) for every entry")
        L.append("  template <typename T, class Out>")
        L.append("  __device__ static __forceinline__ void lu_unpack(const T* J, Out&& out)")
        L.append("  {")
        for r in range(n):
            for c in range(n):
                L.append(f"    out({r * n + c}, {f'J[{lus.pos[(r, c)]}]' if lus.nz(r, c) else 'T(0.0)'});")
        L.append("  }")
        if self.jac is not None:
            L.append("  // analytic Jacobian d f_i / d y_j (every path through the intermediates once)")
            L.append("  // into the packed layout, in the split form")
            L.append("  template <typename T, class A>")
            L.append(f"  __device__ static __forceinline__ void jacobian({sig}, A J)")
            L.append("  {")
            L += I4(head + jac_lines)
            L.append("    (void)time; (void)P; (void)PD; (void)F;")
            L.append("  }")
        L.append("")
        return L

    def metadata_json(self) -> str:
        return json.dumps(self.metadata(), indent=1)
