"""goss objects -> goss_b200 objects, for a backend switch inside goss itself.

goss's Python entry points build a ``goss.ParameterizedODE`` (from a ``.ode``
file through gotran), a solver from ``goss.solvers`` and a
``goss.ODESystemSolver`` (reference ``python/goss/ode.py:144-166``,
``solvers.py:13-214``, ``systemsolver.py:15-134``).  These functions make the
goss_b200 counterparts of such objects, carrying over what the user set on
them: field states, field parameters and monitored intermediates of the model,
its current parameter values, the solver class, its parameters and internal
time step.  goss's model objects do not keep the ``.ode`` source they were
compiled from, so the caller passes it (a path or a parsed model).

The objects are only read through their public goss API (duck typing), so
nothing here imports goss.
"""
from __future__ import annotations

from typing import Any, Optional

from .ode import ParameterizedODE
from .solvers import solver_mapper
from .systemsolver import ODESystemSolver


def ode_from_goss(ode: Any, source: Any, code_params: Optional[dict] = None) -> ParameterizedODE:
    """goss_b200 model of a goss ``ParameterizedODE`` compiled from ``source``."""
    b = ParameterizedODE(source, field_states=list(ode.field_state_names),
                         field_parameters=list(ode.field_parameter_names),
                         monitored=list(ode.monitored_names), code_params=code_params)
    for name, value in dict(ode.parameters).items():
        b.set_parameter(name, float(value))
    return b


def solver_from_goss(solver: Any, ode: ParameterizedODE):
    """The goss_b200 solver of the same class as a goss solver, with its
    parameters and internal time step, attached to ``ode``."""
    name = type(solver).__name__
    if name not in solver_mapper:
        raise TypeError(f"{name} has no goss_b200 counterpart (available: {sorted(solver_mapper)})")
    s = solver_mapper[name](ode)
    s.update_parameters(dict(solver.parameters))
    s.internal_time_step = float(solver.internal_time_step)
    return s


def system_from_goss(num_nodes: int, solver: Any, ode: Any, source: Any, precision: str = "double",
                     device: int = 0, code_params: Optional[dict] = None) -> ODESystemSolver:
    """A goss_b200 ``ODESystemSolver`` in place of
    ``goss.ODESystemSolver(num_nodes, solver, ode)``."""
    bode = ode_from_goss(ode, source, code_params)
    return ODESystemSolver(int(num_nodes), solver_from_goss(solver, bode), bode, precision=precision, device=device)
