"""The goss Python API surface that needs no GPU work.

Ported from the reference's ``tests/test_parameterized_ode_bindings.py`` and
``tests/test_ode_solver_bindings.py`` (constructors, names, parameters,
solver parameter handling and errors).
"""
from __future__ import annotations

import numpy as np
import pytest

import goss_b200 as goss


@pytest.fixture(scope="module")
def oscilator():
    return goss.ParameterizedODE("oscilator")


@pytest.mark.parametrize("field_states, field_state_indices",
                         [([], []), (["x"], [0]), (["y"], [1]), (["x", "y"], [0, 1]), (["y", "x"], [1, 0])])
def test_parameterized_ode_field_states(field_states, field_state_indices):
    ode = goss.ParameterizedODE("oscilator", field_states=field_states)
    assert ode.num_field_states == len(field_states)
    assert ode.field_state_names == field_states
    assert ode.num_states == 2
    assert ode.num_field_parameters == 0
    assert ode.num_parameters == 2
    assert ode.num_monitored == 0
    assert ode.state_names == ["x", "y"]
    assert ode.parameter_names == ["a", "b"]
    assert ode.field_state_indices == field_state_indices
    assert ode.field_parameter_names == []
    assert ode.monitored_names == []


@pytest.mark.parametrize("field_parameters", [[], ["a", "b"]])
def test_parameterized_ode_field_parameters(field_parameters):
    ode = goss.ParameterizedODE("oscilator", field_parameters=field_parameters)
    assert ode.num_field_parameters == len(field_parameters)
    assert ode.field_parameter_names == field_parameters


def test_parameterized_ode_parameters(oscilator):
    ode = oscilator.copy()
    assert ode.get_parameter("a") == 1.0 and ode.get_parameter("b") == 1.0
    ode.set_parameter("a", 42.0)
    ode.set_parameter("b", 13.0)
    assert ode.parameters == {"a": 42.0, "b": 13.0}
    assert oscilator.get_parameter("a") == 1.0  # copies are independent
    with pytest.raises(RuntimeError):
        ode.set_parameter("nope", 1.0)


def test_parameterized_ode_constructors(oscilator):
    ode_new = goss.ParameterizedODE(num_states=3, num_parameters=1)
    assert ode_new.num_states == 3 and ode_new.num_parameters == 1
    assert oscilator.copy().num_states == 2
    with pytest.raises(ValueError):
        goss.ODE(42)
    with pytest.raises(FileNotFoundError):
        goss.ParameterizedODE("no_such_model")


def test_invalid_field_names():
    with pytest.raises(ValueError):
        goss.ParameterizedODE("oscilator", field_states=["a"])


def test_state_and_ic(oscilator):
    assert np.allclose(oscilator.get_ic(), [1.0, 0.0])
    assert oscilator.is_dae is False


@pytest.mark.parametrize("Solver", goss.solvers.GOSSSolvers)
def test_solver_constructors(Solver, oscilator):
    cls = goss.solvers.solver_mapper[Solver.name]
    assert cls(oscilator).num_states == 2
    s = cls()
    assert s.num_states == 0
    s.attach(oscilator)
    assert s.num_states == 2
    assert s.get_ode() is oscilator


def test_invalid_argument_constructor():
    with pytest.raises(ValueError):
        goss.solvers.ExplicitEuler("invalid_argument")


@pytest.mark.parametrize("Solver", goss.solvers.GOSSNonAdaptiveSolvers)
def test_is_adaptive_false(Solver):
    assert goss.solvers.solver_mapper[Solver.name]().is_adaptive is False


@pytest.mark.parametrize("Solver", goss.solvers.GOSSAdaptiveSolvers)
def test_is_adaptive_true(Solver):
    assert goss.solvers.solver_mapper[Solver.name]().is_adaptive is True


@pytest.mark.parametrize("Solver", goss.solvers.GOSSSolvers)
def test_set_and_update_parameters(Solver):
    cls = goss.solvers.solver_mapper[Solver.name]
    solver = cls()
    parameters = solver.parameters
    new = {}
    for name, default_value in cls.default_parameters().items():
        if isinstance(default_value, bool):
            new[name] = not parameters[name]
        elif isinstance(default_value, int):
            new[name] = 42
        else:
            new[name] = 42.0
    for name, value in new.items():
        solver.set_parameter(name, value)
        assert np.isclose(solver.parameters[name], value)
    solver2 = cls()
    solver2.update_parameters(new)
    for name, value in new.items():
        assert np.isclose(solver2.get_parameter(name), value)


def test_set_invalid_parameters():
    solver = goss.solvers.ThetaSolver()
    with pytest.raises(TypeError):
        solver.set_parameter("theta", "hello")
    with pytest.raises(KeyError):
        solver.set_parameter("invalid_parameter", 42.0)


def test_repr_str_and_internal_time_step():
    solver = goss.solvers.ESDIRK23a()
    assert str(solver) == "ESDIRK23a"
    assert repr(solver) == "ESDIRK23a()"
    solver.internal_time_step = 0.42
    assert np.isclose(solver.internal_time_step, 0.42)


def test_adaptive_methods(oscilator):
    solver = goss.solvers.ESDIRK23a(oscilator)
    solver.reset()
    assert solver.nfevals == 0 and solver.ndtsa == 0 and solver.ndtsr == 0
    solver.get_num_accepted()
    solver.get_num_rejected()
    assert solver.get_current_time() == 0.0
    solver.set_tol(atol=1e-5, rtol=1e-4)
    assert solver.atol == 1e-5 and solver.rtol == 1e-4
    solver.set_iord(42)
    assert solver.iord == 42


@pytest.mark.parametrize("Solver", goss.solvers.GOSSImplicitSolvers)
def test_num_jac_comp_starts_at_zero(Solver, oscilator):
    assert goss.solvers.solver_mapper[Solver.name](oscilator).num_jac_comp() == 0


def test_has_openmp():
    assert goss.has_openmp() is True


def test_c_params_layout():
    s = goss.solvers.ThetaSolver()
    s.set_parameter("theta", 0.75)
    s.internal_time_step = 0.05
    p = s.c_params()
    assert p.theta == 0.75 and p.ldt == 0.05 and p.max_iterations == 30


def test_solver_trace_rejects_solvers_without_adjoint():
    from goss_b200.adjoint import SolverTrace

    ode = goss.ParameterizedODE("fitzhughnagumo", field_parameters=["a", "b"])
    with pytest.raises(ValueError):
        SolverTrace(ode, 4, 1.0, 10, 2, 10, solver="ThetaSolver")


def test_get_field_states_into_a_caller_array_checks_its_shape():
    import goss_b200 as goss

    ode = goss.ParameterizedODE("oscilator", field_states=["x"])
    with pytest.raises(ValueError):
        # the check precedes any device work
        goss.ODESystemSolver.get_field_states(
            type("S", (), {"_num_nodes": 4, "_ode": ode})(), out=np.zeros((3, 1)))


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the behaviour without a GPU")
def test_without_a_gpu_the_system_fails_loudly():
    # no CPU path stands behind the API: without a device the runtime's first
    # CUDA call raises
    import goss_b200 as goss
    from goss_b200._capi import GossError

    ode = goss.ParameterizedODE("oscilator")
    with pytest.raises(GossError, match="CUDA"):
        goss.ODESystemSolver(4, goss.solvers.GRL1(ode), ode)


def test_missing_runtime_library_raises(monkeypatch, tmp_path):
    from goss_b200 import _capi

    monkeypatch.setattr(_capi, "RUNTIME_SO", tmp_path / "libgoss_b200.so")
    monkeypatch.setattr(_capi, "_lib", None)
    with pytest.raises(_capi.ExtensionMissingError, match="is missing"):
        _capi.lib()
