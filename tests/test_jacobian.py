"""Analytic Jacobian (``code_params={"generate_jacobian": True}``) and the
structure-aware Newton linear algebra of the implicit kernels, on the CPU.

* The generated analytic Jacobian is the plugin's ``compute_jacobian``
  override the reference generates (``python/goss/codegeneration.py:622-641``);
  the oracle's copy of it equals the plugin's bit for bit inside the
  reference's compiled ``ODE`` and agrees with the reference's forward
  differences (``ODE.cpp:47-67``) to their truncation error.
* The implicit solvers driven by it (reference ThetaSolver, ImplicitEuler,
  ESDIRK23a with the plugin) equal the oracle's restatement bit for bit.
* The packed LU and substitution the kernels run (codegen/sparse.py) equal
  the reference's dense ``ODE::lu_factorize`` / ``forward_backward_subst``
  bit for bit on matrices with the model's Jacobian structure.
"""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from goss_b200.codegen.sparse import LUStructure
from goss_b200.compilemodule import code_params_jacobian
from helpers import meta, oracle_model, perturbed_states, ref_system, variant_dir

TT04, FPS = "tentusscher_2004_mcell", ("g_Kr", "g_CaL")


def _exec_lines(lines, env):
    """Run generated C statements of the forms codegen/sparse.py prints
    (assignments, ``-=``, blocks) with Python floats: IEEE double arithmetic
    without fused multiply-adds, as the oracle's C build."""
    for line in lines:
        body = line.strip().strip("{}").replace("const double ", "").replace("double ", "")
        for stmt in body.split(";"):
            stmt = stmt.strip()
            if stmt:
                exec(stmt, {}, env)


def _newton_matrix(struct, rng, h=0.1):
    n = len(struct)
    J = np.where(np.array(struct, dtype=bool), rng.standard_normal((n, n)), 0.0)
    return np.ascontiguousarray(np.eye(n) - h * J)


@pytest.mark.parametrize("name", ["tentusscher_2004_mcell", "tentusscher_panfilov_2006_M_cell",
                                  "beeler_reuter_1977", "fitzhughnagumo"])
def test_packed_lu_and_solve_bit_identical_to_dense(name):
    md = meta(variant_dir(name))
    lus = LUStructure(md["jacobian_structure"])
    assert lus.nnz == md["lu_nnz"]
    om = oracle_model(name)
    rng = np.random.default_rng(5)
    for trial in range(20):
        A = _newton_matrix(lus.jac, rng, h=0.05 * (trial + 1))
        dense = A.copy()
        om.lu_factorize(dense)
        J = [0.0] * lus.nnz
        for (r, c), k in lus.pos.items():
            J[k] = float(A[r, c])
        env = {"J": J}
        _exec_lines(lus.lu_factorize_lines(), env)
        for (r, c), k in lus.pos.items():
            assert J[k] == dense[r, c], (r, c, J[k], dense[r, c])
        outside = [dense[r, c] for r in range(lus.n) for c in range(lus.n) if not lus.nz(r, c)]
        assert not np.any(outside)  # the dense factors stay 0 outside the structure
        b = rng.standard_normal(lus.n)
        x_dense = om.forward_backward_subst(dense, b)
        x = [0.0] * lus.n
        _exec_lines(lus.solve_lines(), {"J": J, "b": [float(v) for v in b], "x": x})
        assert np.array_equal(np.array(x), x_dense)
        # b and x may be the same array (ESDIRK23a's error estimate)
        y = [float(v) for v in b]
        _exec_lines(lus.solve_lines("J", "y", "y"), {"J": J, "y": y})
        assert np.array_equal(np.array(y), x_dense)


def test_dense_reference_lu_matches_oracle():
    r = ref_system(TT04, "ThetaSolver", 1)
    if r is None:
        pytest.skip("reference plugin not built")
    lus = LUStructure(meta(variant_dir(TT04))["jacobian_structure"])
    om = oracle_model(TT04)
    rng = np.random.default_rng(2)
    A = _newton_matrix(lus.jac, rng)
    a, b = A.copy(), A.copy()
    om.lu_factorize(a)
    r.lu_factorize(b)
    assert np.array_equal(a, b)
    rhs = rng.standard_normal(lus.n)
    assert np.array_equal(om.forward_backward_subst(a, rhs), r.forward_backward_subst(b, rhs))


@pytest.mark.parametrize("name", ["tentusscher_2004_mcell", "tentusscher_panfilov_2006_M_cell",
                                  "beeler_reuter_1977"])
def test_forward_difference_jacobian_is_zero_outside_the_structure(name):
    md = meta(variant_dir(name))
    S = np.array(md["jacobian_structure"], dtype=bool)
    om = oracle_model(name)
    rng = np.random.default_rng(4)
    for y in perturbed_states(om.ic, 5, rng, 0.05):
        jac = om.jacobian(y, 3.0)
        assert not np.any(jac[~S])


def test_analytic_jacobian_close_to_forward_differences():
    ana = oracle_model(TT04, FPS, True)
    fd = oracle_model(TT04, FPS)
    rng = np.random.default_rng(8)
    S = np.array(meta(variant_dir(TT04, FPS, True))["jacobian_structure"], dtype=bool)
    for y in perturbed_states(ana.ic, 6, rng, 0.05):
        Ja, Jf = ana.jacobian(y, 1.0), fd.jacobian(y, 1.0)
        assert not np.any(Ja[~S])
        scale = np.maximum(np.abs(Jf).max(axis=1, keepdims=True), 1e-300)
        assert np.max(np.abs(Ja - Jf) / scale) < 1e-5
        # the diagonal is the exact-rule linearisation (the gotran rule double
        # counts some paths, so compare with the exact variant's own formula)
        central = np.zeros_like(Ja)
        for j in range(len(y)):
            h = 1e-6 * max(abs(y[j]), 1e-3)
            yp, ym = y.copy(), y.copy()
            yp[j] += h
            ym[j] -= h
            central[:, j] = (ana.rhs(yp, 1.0) - ana.rhs(ym, 1.0)) / (2 * h)
        assert np.max(np.abs(Ja - central) / scale) < 1e-6


def test_analytic_jacobian_bit_identical_to_reference_plugin():
    r = ref_system(TT04, "ThetaSolver", 1, FPS, jacobian=True)
    if r is None:
        pytest.skip("reference plugin not built")
    om = oracle_model(TT04, FPS, True)
    rng = np.random.default_rng(12)
    for y in perturbed_states(om.ic, 4, rng, 0.05):
        assert np.array_equal(om.jacobian(y, 2.0), r.compute_jacobian(y, 2.0))


@pytest.mark.parametrize("solver,steps,ldt", [
    ("ThetaSolver", 100, 0.1),
    ("ImplicitEuler", 100, 0.1),
    ("ESDIRK23a", 40, -1.0),
])
def test_implicit_solvers_with_analytic_jacobian_bit_identical_to_reference(solver, steps, ldt):
    om = oracle_model(TT04, FPS, True)
    r = ref_system(TT04, solver, 3, FPS, jacobian=True, ldt=ldt)
    if r is None:
        pytest.skip("reference plugin not built")
    rng = np.random.default_rng(21)
    y0 = perturbed_states(om.ic, 3, rng, 0.02)
    md = meta(variant_dir(TT04, FPS, True))
    defaults = np.array([md["default_parameters"][i] for i in md["field_parameter_indices"]])
    fp = defaults[None, :] * (1 + rng.uniform(-0.05, 0.05, (3, 2)))
    o = pyoracle.OracleSystem(om, solver, 3, ldt=ldt)
    o.states[:] = y0
    o.field_params[:] = fp
    r.set_states(y0)
    r.set_field_parameters(fp)
    for k in range(steps):
        assert o.forward(k * 0.1, 0.1) == 0
        assert r.forward(k * 0.1, 0.1) == 0
    assert np.array_equal(o.states, r.get_states())
    jc, _, _ = o.counters()
    assert np.array_equal(jc, r.num_jac_comp())


def test_code_params_validation():
    assert code_params_jacobian(None) is False
    assert code_params_jacobian({}) is False
    assert code_params_jacobian({"generate_jacobian": True}) is True
    # the reference test's full option set (tests/test_codegeneration.py:5-13)
    assert code_params_jacobian({"state_repr": "named", "body_repr": "named", "use_cse": False,
                                 "generate_forward_backward_subst": True, "generate_jacobian": True,
                                 "generate_lu_factorization": True, "optimize_exprs": "numerals"}) is True
    assert code_params_jacobian({"some_unknown_option": 3}) is False
    with pytest.raises(ValueError):
        code_params_jacobian({"state_repr": "list"})
    with pytest.raises(ValueError):
        code_params_jacobian({"generate_jacobian": "yes"})
    with pytest.raises(TypeError):
        code_params_jacobian(["generate_jacobian"])


def test_jacobian_variant_is_its_own_variant():
    plain, ana = variant_dir(TT04, FPS), variant_dir(TT04, FPS, True)
    assert plain != ana
    assert meta(ana)["jacobian"] and not meta(plain)["jacobian"]
    assert meta(ana)["lu_nnz"] == meta(plain)["lu_nnz"] == 71
    assert "compute_jacobian" in (ana / "goss_plugin.h").read_text()
    assert "compute_jacobian" not in (plain / "goss_plugin.h").read_text()
    assert "has_jacobian = true" in (ana / "device.cuh").read_text()
