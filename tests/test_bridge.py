"""goss_b200.bridge: goss objects -> goss_b200 objects (a backend switch
inside goss).  goss itself is not importable here (gotran and cppyy are
absent), so stand-ins expose the public goss API the bridge reads
(python/goss/ode.py:205-230, solvers.py:84-125)."""
from __future__ import annotations

import numpy as np
import pytest

from goss_b200 import bridge


class _GossODE:  # goss.ParameterizedODE's public attributes
    def __init__(self, parameters, field_states=(), field_parameters=(), monitored=()):
        self.parameters = dict(parameters)
        self.field_state_names = list(field_states)
        self.field_parameter_names = list(field_parameters)
        self.monitored_names = list(monitored)


class ThetaSolver:  # named like goss.solvers.ThetaSolver
    def __init__(self):
        self.parameters = {"eta_0": 1.0, "kappa": 0.1, "relative_tolerance": 1e-12, "max_iterations": 30,
                           "max_relative_previous_residual": 0.01, "always_recompute_jacobian": False,
                           "num_refinements_without_always_recomputing_jacobian": 2, "min_dt": 0.0001,
                           "theta": 0.75}
        self.internal_time_step = 0.05


class GRL1:
    parameters = {"delta": 1e-8}
    internal_time_step = 0.01


class BasicImplicitEuler:
    parameters = {}
    internal_time_step = 0.1


def test_model_and_solver_carry_over():
    gode = _GossODE({"g_Kr": 0.2, "g_CaL": 1.9e-4}, field_states=["V"], field_parameters=["g_Kr", "g_CaL"])
    ode = bridge.ode_from_goss(gode, "tentusscher_2004_mcell")
    assert ode.field_parameter_names == ["g_Kr", "g_CaL"]
    assert ode.field_state_names == ["V"]
    assert ode.get_parameter("g_Kr") == 0.2 and ode.get_parameter("g_CaL") == 1.9e-4
    s = bridge.solver_from_goss(ThetaSolver(), ode)
    assert type(s).__name__ == "ThetaSolver" and s.get_ode() is ode
    assert s.get_parameter("theta") == 0.75 and s.internal_time_step == 0.05
    with pytest.raises(TypeError):
        bridge.solver_from_goss(BasicImplicitEuler(), ode)


@pytest.mark.gpu
def test_system_from_goss_matches_oracle():
    import pyoracle
    from helpers import oracle_model, parity, perturbed_states

    name = "tentusscher_panfilov_2006_M_cell"
    om = oracle_model(name)
    params = dict(zip(bridge.ParameterizedODE(name).parameter_names, om.default_params))
    params["g_Kr"] *= 1.3
    system = bridge.system_from_goss(24, GRL1(), _GossODE(params, field_states=["V"]), name)
    y0 = perturbed_states(om.ic, 24, np.random.default_rng(3), 0.05)
    system.set_states(y0)
    o = pyoracle.OracleSystem(om, "GRL1", 24, ldt=0.01)
    o.states[:] = y0
    o.params[: om.np] = [params[p] for p in system.ode.parameter_names]
    for k in range(15):
        system.forward(float(k), 1.0)
        o.forward(float(k), 1.0)
    assert parity(system.states, o.states, rtol=1e-10) <= 1.0
