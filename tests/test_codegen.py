"""Front end and code generator, pinned against the reference's golden vectors.

CPU only: the generated C restatement of each model (the oracle's model
code, printed from the same programs as the CUDA device code) is evaluated
and compared with

* gotran's generated goss classes shipped by the reference
  (``cpp/tests/fhn.h``, ``cpp/tests/beeler_reuter_1977.h``, ``tests/oscilator.h``),
* gotran's generated numpy rhs of the TP06 M-cell model
  (``benchmarks/tentusscher_panfilov_2006_M_cell.py``),

through the fixtures in ``tests/golden`` (``make_golden.py``).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest
import sympy as sp

from goss_b200.codegen.ir import ModelIR
from goss_b200.codegen.odeparse import ODEParseError, parse_ode_text
from goss_b200.codegen.variant import write_variant
from helpers import GOLDEN, meta, oracle_model, variant_dir

import pyoracle

# the reference source tree (GOSS_REFERENCE or the oracle recipe's REF); the
# tests that regenerate from its .ode files skip where it is absent
REF = pyoracle.reference_dir() or Path("/nonexistent-reference")


def test_state_order_follows_derivatives_and_parameters_sorted():
    text = """
parameters("A", zeta=1.0, alpha=2.0, Beta=3.0)
states(x=1.0, y=2.0, z=3.0)
parameters("B", c=4.0)
dz_dt = -z
dx_dt = alpha*x
dy_dt = zeta*y + c + Beta
"""
    m = parse_ode_text(text, "toy")
    assert m.state_names == ["z", "x", "y"]
    assert m.parameter_names == ["Beta", "alpha", "zeta", "c"]
    assert list(m.states.values()) == [3.0, 1.0, 2.0]


def test_continuous_conditional_is_logistic():
    m = parse_ode_text("parameters(s=1.0)\nstates(v=0.0)\n"
                       "dv_dt = ContinuousConditional(Ge(time, s), 1, 0, 0.2)\n", "cc")
    e = m.derivatives["v"]
    t = sp.Symbol("time", real=True)
    f = sp.lambdify([t, m.sym("s")], e)
    assert f(1.0, 1.0) == pytest.approx(0.5)
    assert f(3.0, 1.0) == pytest.approx(1.0, abs=1e-4)
    assert f(-1.0, 1.0) == pytest.approx(0.0, abs=1e-4)


@pytest.mark.parametrize("bad", [
    "states(x=1)\n",                              # no derivative
    "states(x=1)\ndx_dt = foo(x)\n",              # unknown function
    "states(x=1)\ndx_dt = y\n",                   # undefined symbol
    "states(x=1)\ndx_dt = x\ndx_dt = 2*x\n",      # derivative twice
    "states(x=1)\nimport os\ndx_dt = x\n",        # statements outside the DSL
])
def test_parse_errors(bad):
    with pytest.raises(ODEParseError):
        parse_ode_text(bad, "bad")


def _cpp_fixture(name):
    return np.load(GOLDEN / f"{name}_cpp_fixture.npz")


@pytest.mark.parametrize("name", ["fhn", "beeler_reuter_1977", "oscilator"])
def test_generated_model_matches_gotran_fixture(name):
    """eval, linearized_eval and the linear-term flags of the generated model
    equal gotran's generated class on 64 seeded states."""
    g = _cpp_fixture(name)
    om = oracle_model(name)
    md = meta(variant_dir(name))
    assert list(g["linear_terms"]) == md["linear_terms"]
    p = g["params"]
    for y, t, ev, lrhs, lin in zip(g["states"], g["times"], g["eval"], g["lin_rhs"], g["linear"]):
        np.testing.assert_allclose(om.rhs(y, t, p), ev, rtol=1e-11, atol=1e-13)
        l, r = om.linearized(y, t, p)
        np.testing.assert_allclose(r, lrhs, rtol=1e-11, atol=1e-13)
        np.testing.assert_allclose(l, lin, rtol=1e-11, atol=1e-13)


def test_generated_tp06_rhs_matches_gotran_numpy():
    g = np.load(GOLDEN / "tp06_numpy_fixture.npz")
    md = meta(variant_dir("tentusscher_panfilov_2006_M_cell"))
    assert list(g["state_order"]) == md["state_names"]
    assert list(g["param_order"]) == md["parameter_names"]
    om = oracle_model("tentusscher_panfilov_2006_M_cell")
    for y, t, v in zip(g["states"], g["times"], g["values"]):
        np.testing.assert_allclose(om.rhs(y, t, g["params"]), v, rtol=1e-11, atol=1e-14)


def test_gotran_linearization_counts_conditional_chain_twice():
    """The fixture's linear[7] of Beeler-Reuter is reproduced only with the
    gotran rule; the exact rule differs by the chain through V_eff_1."""
    if not (REF / "cpp/tests/beeler_reuter_1977.ode").exists():
        pytest.skip("reference sources not available")
    from goss_b200.codegen.odeparse import load_ode

    m = load_ode(REF / "cpp/tests/beeler_reuter_1977.ode")
    exact = ModelIR(m, linearization="exact").linearized_program(split=False)
    gotran = ModelIR(m, linearization="gotran").linearized_program(split=False)
    ex = {o.index: o.expr for o in exact.outputs() if o.array == "linear"}
    go = {o.index: o.expr for o in gotran.outputs() if o.array == "linear"}
    assert set(ex) == set(go)
    differing_derivs = {a.name for a in gotran.assigns()} ^ {a.name for a in exact.assigns()}
    same = {a.name: sp.srepr(a.expr) for a in exact.assigns()}
    changed = [a.name for a in gotran.assigns() if a.name in same and same[a.name] != sp.srepr(a.expr)]
    assert changed == ["di_K1_dV"] and not differing_derivs


def test_shipped_variants_regenerate_identically(tmp_path):
    """The committed generated sources are what the generator writes today."""
    if not REF.is_dir():
        pytest.skip("reference sources not available")
    from goss_b200 import models
    from goss_b200.codegen.odeparse import load_ode
    from goss_b200.codegen.variant import variant_id

    for entry in models.SHIPPED:
        model = load_ode(REF / entry["ode"])
        mon = entry.get("monitored", [])
        ident = variant_id(model, entry["field_parameters"], mon)
        write_variant(model, tmp_path / ident, field_parameters=entry["field_parameters"], monitored=mon)
        for f in ("device.cuh", "module.cu", "oracle_model.c", "goss_plugin.h", "model.json"):
            assert (tmp_path / ident / f).read_text() == (models.HERE / ident / f).read_text(), (ident, f)


def test_op_census_present():
    md = meta(variant_dir("tentusscher_panfilov_2006_M_cell"))
    lin = md["op_census"]["linearized"]
    assert lin["exp"] > 50 and lin["mul"] > 100
    assert md["op_census"]["rhs"]["exp"] > 0
