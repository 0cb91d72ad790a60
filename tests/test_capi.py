"""The C ABI library: it loads, exports every declared entry point, and the
model modules expose descriptors that match their metadata.  No GPU work."""
from __future__ import annotations

import ctypes as C
import json
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from goss_b200 import _capi, models
from goss_b200.compilemodule import load_variant
from helpers import ROOT, oracle_model

HEADER = ROOT / "include" / "goss_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"GOSS_API\s+[\w\s\*]+?\b(goss_\w+)\s*\(", text)))


def test_header_declarations_are_bound():
    assert declared_functions() == _capi.EXPORTED


def test_library_exports_every_declared_symbol():
    L = _capi.lib()
    for name in declared_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(_capi.RUNTIME_SO)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (goss_\w+)", out))
    assert set(declared_functions()) <= exported
    assert L.goss_abi_version() == _capi.ABI_VERSION


def test_default_solver_params_match_reference():
    sp = _capi.SolverParams()
    assert _capi.lib().goss_solver_default_params(_capi.GOSS_THETA, C.byref(sp)) == 0
    assert (sp.ldt, sp.eta_0, sp.kappa, sp.relative_tolerance, sp.max_iterations) == (-1.0, 1.0, 0.1, 1e-12, 30)
    assert (sp.max_relative_previous_residual, sp.min_dt, sp.theta) == (0.01, 0.0001, 0.5)
    assert sp.num_refinements_without_always_recomputing_jacobian == 2
    _capi.lib().goss_solver_default_params(_capi.GOSS_ESDIRK23A, C.byref(sp))
    assert sp.min_dt == 0.001
    _capi.lib().goss_solver_default_params(_capi.GOSS_GRL1, C.byref(sp))
    assert sp.delta == 1e-8
    assert _capi.lib().goss_solver_default_params(99, C.byref(sp)) == _capi.GOSS_ERR_ARGUMENT


@pytest.mark.parametrize("vdir", models.variant_dirs(), ids=lambda p: p.name)
def test_model_descriptor_matches_metadata(vdir):
    mod = load_variant(vdir)
    d = mod.desc.contents
    md = json.loads((vdir / "model.json").read_text())
    assert d.abi_version == _capi.ABI_VERSION
    assert d.name.decode() == md["name"]
    n, npar, nfp = d.num_states, d.num_parameters, d.num_field_parameters
    assert [d.state_names[i].decode() for i in range(n)] == md["state_names"]
    assert [d.parameter_names[i].decode() for i in range(npar)] == md["parameter_names"]
    assert [d.field_parameter_names[i].decode() for i in range(nfp)] == md["field_parameter_names"]
    assert [d.field_parameter_indices[i] for i in range(nfp)] == md["field_parameter_indices"]
    assert [d.initial_conditions[i] for i in range(n)] == md["initial_conditions"]
    assert [d.default_parameters[i] for i in range(npar)] == md["default_parameters"]
    assert [d.linear_terms[i] for i in range(n)] == md["linear_terms"]
    assert d.supported_solvers == (1 << 10) - 1
    assert d.solver_state_rows(_capi.GOSS_GRL1) == 0
    assert d.lu_nnz == md["lu_nnz"] and d.has_jacobian == int(md["jacobian"])
    assert d.solver_state_rows(_capi.GOSS_ESDIRK23A) == 9 + 2 * md["lu_nnz"]
    assert d.solver_state_rows(_capi.GOSS_IMPLICIT_EULER) == 7 + md["lu_nnz"]


def test_host_lu_matches_oracle():
    om = oracle_model("tentusscher_2004_mcell")
    jac = om.jacobian(om.ic, 0.0)
    a = np.ascontiguousarray(np.eye(om.n) - 0.05 * jac)
    b = a.copy()
    assert _capi.lib().goss_lu_factorize(om.n, _capi.ptr(a)) == 0
    om.lib.oracle_lu_factorize(om.n, b.ctypes.data_as(C.POINTER(C.c_double)))
    assert np.array_equal(a, b)
    rhs = np.linspace(-1, 1, om.n)
    x1, x2 = np.zeros(om.n), np.zeros(om.n)
    _capi.lib().goss_forward_backward_subst(om.n, _capi.ptr(a), _capi.ptr(rhs), _capi.ptr(x1))
    om.lib.oracle_forward_backward_subst(om.n, b.ctypes.data_as(C.POINTER(C.c_double)),
                                         rhs.ctypes.data_as(C.POINTER(C.c_double)),
                                         x2.ctypes.data_as(C.POINTER(C.c_double)))
    assert np.array_equal(x1, x2)
