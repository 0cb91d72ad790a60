"""Generate the source tree of one compiled model variant.

A *variant* is one ``.ode`` model combined with the code-generation choices
that change the compiled code: the field parameters (read per node instead of
from the uniform parameter block), the monitored intermediates, the
linearisation rule and whether the analytic Jacobian is generated (the
reference's ``code_params["generate_jacobian"]``).  Its directory holds

``model.json``        names, defaults, linear-term flags, op census
``device.cuh``        CUDA ``__device__`` model (templated on T)
``module.cu``         sm_100a kernels instantiated for the model + the
                      ``goss_model_desc`` factory ``goss_b200_model_<ident>()``
``oracle_model.c``    C restatement used by the CPU oracle (test infrastructure)
``goss_plugin.h``     goss::ParameterizedODE plugin for the reference solvers
                      (test infrastructure)

This replaces the reference's JIT path, ``GossCodeGenerator.file_code()`` +
``cppyy.cppdef`` (``python/goss/compilemodule.py:63-117``).
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path
from typing import Dict, Optional, Sequence

from .emit import ModelSource, c_ident, model_class_name
from .ir import ModelIR
from .odeparse import ODEModel

GENERATOR_VERSION = "8"

_CENSUS_KEYS = ("add", "mul", "div", "exp", "log", "sqrt", "pow", "cmp", "misc")


def _key(field_parameters, monitored, linearization, jacobian) -> list:
    key = [list(field_parameters), list(monitored), linearization]
    return key + [{"jacobian": True}] if jacobian else key


def variant_id(model: ODEModel, field_parameters: Sequence[str] = (), monitored: Sequence[str] = (),
               linearization: str = "gotran", jacobian: bool = False) -> str:
    base = c_ident(model.name)
    if not field_parameters and not monitored and linearization == "gotran" and not jacobian:
        return base
    key = json.dumps(_key(field_parameters, monitored, linearization, jacobian))
    return f"{base}__{hashlib.sha1(key.encode()).hexdigest()[:8]}"


def model_hash(model: ODEModel, field_parameters, monitored, linearization, jacobian: bool = False) -> str:
    h = hashlib.sha1()
    h.update(GENERATOR_VERSION.encode())
    h.update(model.signature().encode())
    h.update(json.dumps(_key(field_parameters, monitored, linearization, jacobian)).encode())
    return h.hexdigest()


def _cstr_list(name: str, items) -> str:
    if not items:
        return f"static const char* const {name}[1] = {{nullptr}};"
    return f"static const char* const {name}[{len(items)}] = {{" + ", ".join(f'"{s}"' for s in items) + "};"


def _num_list(ctype: str, name: str, items, fmt=str) -> str:
    items = list(items)
    if not items:
        return f"static const {ctype} {name}[1] = {{0}};"
    return f"static const {ctype} {name}[{len(items)}] = {{" + ", ".join(fmt(v) for v in items) + "};"


def device_struct(ident: str) -> str:
    """Name of a variant's device model struct (unique per variant)."""
    return f"M_{ident}"


def emit_module(src: ModelSource, ident: str) -> str:
    md = src.metadata()
    cls = device_struct(ident)
    from .printer import c_double

    lines = [
        f"// Generated by goss_b200.codegen for model '{src.name}' (variant {ident}); do not edit.",
        "// sm_100a solver kernels instantiated for this model and its goss_model_desc factory.",
        '#include "goss_adjoint.cuh"',
        '#include "goss_kernels.cuh"',
        '#include "device.cuh"',
        "",
        "namespace {",
        f"using Model = goss_b200::models::{cls};",
        _cstr_list("state_names", md["state_names"]),
        _cstr_list("parameter_names", md["parameter_names"]),
        _cstr_list("field_parameter_names", md["field_parameter_names"]),
        _num_list("uint32_t", "field_parameter_indices", md["field_parameter_indices"]),
        _num_list("double", "initial_conditions", md["initial_conditions"], c_double),
        _num_list("double", "default_parameters", md["default_parameters"], c_double),
        _num_list("uint8_t", "linear_terms", md["linear_terms"]),
        _num_list("uint32_t", "op_lin", [md["op_census"]["linearized"][k] for k in _CENSUS_KEYS]),
        _num_list("uint32_t", "op_rhs", [md["op_census"]["rhs"][k] for k in _CENSUS_KEYS]),
        "int launch(const goss_launch* L) { return goss_b200::launch_solver<Model>(L); }",
        "int eval(const goss_eval_launch* L) { return goss_b200::launch_eval<Model>(L); }",
        "uint32_t rows(int32_t s) { return goss_b200::solver_state_rows<Model>(s); }",
        "int adjoint(const goss_adjoint_launch* L) { return goss_b200::launch_adjoint<Model>(L); }",
        "}  // namespace",
        "",
        f'extern "C" GOSS_API const goss_model_desc* goss_b200_model_{ident}(void)',
        "{",
        "    static const goss_model_desc d = {",
        "        GOSS_B200_ABI_VERSION,",
        f'        "{src.name}",',
        f"        {len(md['state_names'])}u, {len(md['parameter_names'])}u, {len(md['field_parameter_names'])}u, "
        f"{len(md['monitored_names'])}u,",
        "        state_names, parameter_names, field_parameter_names, field_parameter_indices,",
        "        initial_conditions, default_parameters, linear_terms,",
        "        (1u << GOSS_NUM_SOLVERS) - 1u,",
        "        launch, eval, rows, op_lin, op_rhs, adjoint,",
        f"        {1 if md['jacobian'] else 0}u, {md['lu_nnz']}u,",
        "    };",
        "    return &d;",
        "}",
    ]
    return "\n".join(lines) + "\n"


def write_variant(model: ODEModel, outdir: Path, field_parameters: Sequence[str] = (),
                  monitored: Sequence[str] = (), linearization: str = "gotran",
                  ident: Optional[str] = None, jacobian: bool = False) -> Dict:
    """Write all generated sources of a variant into ``outdir``."""
    ident = ident or variant_id(model, field_parameters, monitored, linearization, jacobian)
    ir = ModelIR(model, field_parameters=field_parameters, monitored=monitored, linearization=linearization)
    src = ModelSource(ir, jacobian=jacobian)
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    md = src.metadata()
    md.update(variant=ident, linearization=linearization,
              hash=model_hash(model, field_parameters, monitored, linearization, jacobian),
              generator_version=GENERATOR_VERSION, class_name=model_class_name(model.name))
    files = {
        "device.cuh": src.emit_device(device_struct(ident)),
        "module.cu": emit_module(src, ident),
        "oracle_model.c": src.emit_oracle_c(),
        "goss_plugin.h": src.emit_goss_plugin(),
        "model.json": json.dumps(md, indent=1) + "\n",
    }
    for name, text in files.items():
        p = outdir / name
        if not p.exists() or p.read_text() != text:
            p.write_text(text)
    return md
