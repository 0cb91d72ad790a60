"""Solver objects of the goss Python API.

Mirrors ``goss.solvers`` (reference ``python/goss/solvers.py:13-491``): the
same class names, default parameters, type checks and error types.  A solver
carries its parameters and the ODE it is attached to; the arithmetic runs in
the sm_100a kernels.  ``forward``/``solve`` on a single state vector run a
one-node :class:`~goss_b200.systemsolver.ODESystemSolver`.

Solvers of the reference outside this package's scope (RKF32,
BasicImplicitEuler, ESDIRK4O32) are not provided.
"""
from __future__ import annotations

import abc
from enum import Enum
from typing import Any, Dict, Optional

import numpy as np

from . import _capi
from .ode import ODE


class ODESolver(abc.ABC):
    """Base class of the solvers (``goss.solvers.ODESolver``)."""

    _kind: int = -1
    _adaptive = False

    def __init__(self, *args, **kwargs):
        self._ode: Optional[ODE] = None
        self._params: Dict[str, Any] = dict(self.__class__.default_parameters())
        self._ldt = -1.0
        self._counters = dict(jac_comp=0, nfevals=0, ndtsa=0, ndtsr=0, accepted=0, rejected=0)
        self._sys = None  # one-node system used by forward()/solve()
        if len(args) == 0:
            pass
        elif isinstance(args[0], ODE):
            self.attach(args[0])
        elif isinstance(args[0], ODESolver):
            other = args[0]
            self._ode = other._ode
            self._params = dict(other._params)
            self._ldt = other._ldt
        else:
            raise ValueError(f"Unknown argument of type {type(args[0])}")

    def __str__(self) -> str:
        return f"{self.__class__.__name__}"

    def __repr__(self) -> str:
        return f"{self.__class__.__name__}()"

    # -- configuration -------------------------------------------------------
    def reset(self) -> None:
        for k in self._counters:
            self._counters[k] = 0
        self._sys = None

    def attach(self, ode: ODE) -> None:
        if ode.is_dae and not isinstance(self, ImplicitODESolver):
            raise RuntimeError("cannot integrate a DAE ode with an explicit solver.")
        self._ode = ode
        self.reset()

    @property
    def is_adaptive(self) -> bool:
        """Flag to indicate whether the solver is adaptive for not"""
        return self._adaptive

    @staticmethod
    def default_parameters() -> Dict[str, Any]:
        """Dictionary with the default parameters"""
        return {}

    def update_parameters(self, parameters: Dict[str, Any]):
        for k, v in parameters.items():
            self.set_parameter(k, v)

    @property
    def internal_time_step(self) -> float:
        """Time step used internally by the solver"""
        return self._ldt

    @internal_time_step.setter
    def internal_time_step(self, time_step: float) -> None:
        self._ldt = float(time_step)

    @property
    def parameters(self) -> Dict[str, Any]:
        return {name: self.get_parameter(name) for name in self.__class__.default_parameters()}

    def get_parameter(self, name: str) -> Any:
        if name not in self._params:
            raise KeyError(f"Invalid parameter {name}")
        return self._params[name]

    def set_parameter(self, name: str, value: Any):
        parameters = self.__class__.default_parameters()
        if name not in parameters:
            raise KeyError(f"Invalid parameter {name}, expected one of {parameters.keys()}")
        if not isinstance(value, type(parameters[name])):
            raise TypeError(f"Expected parameter {name} to be of type{type(parameters[name])}, got {type(value)}")
        self._params[name] = value

    def get_ode(self) -> ODE:
        return self._ode

    def copy(self):
        return self.__class__(self)

    @property
    def num_states(self) -> int:
        return self._ode.num_states if self._ode is not None else 0

    @property
    def kind(self) -> int:
        return self._kind

    def c_params(self) -> _capi.SolverParams:
        """Parameters in the layout of ``goss_solver_params``."""
        sp = _capi.SolverParams()
        _capi.check(_capi.lib().goss_solver_default_params(self._kind, sp))
        sp.ldt = float(self._ldt)
        for k, v in self._params.items():
            if hasattr(sp, k):
                setattr(sp, k, type(getattr(sp, k))(v))
        return sp

    # -- single state vector --------------------------------------------------
    def _one_node(self):
        from .systemsolver import ODESystemSolver

        if self._ode is None:
            raise RuntimeError("no ODE attached to the solver")
        if self._sys is None:
            self._sys = ODESystemSolver(1, self, self._ode)
        return self._sys

    def forward(self, y: np.ndarray, t: float, interval: float):
        """Advance the state vector ``y`` in place by ``interval``."""
        sys = self._one_node()
        sys._set_states(np.asarray(y, dtype=np.float64).reshape(1, -1))
        sys.forward(t, interval)
        y[:] = sys.states[0]

    def solve(self, t: np.ndarray, y0: Optional[np.ndarray] = None) -> np.ndarray:
        """States at every time of ``t`` starting from ``y0`` (default: the IC)."""
        if y0 is None:
            y0 = self.get_ode().get_ic()
        t = np.asarray(t, dtype=np.float64)
        y = np.zeros((t.size, self.num_states))
        y[0, :] = y0
        cur = np.array(y0, dtype=np.float64)
        for it in range(1, t.size):
            self.forward(cur, t[it - 1], t[it] - t[it - 1])
            y[it, :] = cur
        return y


class ExplicitEuler(ODESolver):
    _kind = _capi.GOSS_EXPLICIT_EULER


class RL1(ODESolver):
    _kind = _capi.GOSS_RL1


class RL2(ODESolver):
    _kind = _capi.GOSS_RL2


class RK2(ODESolver):
    _kind = _capi.GOSS_RK2


class RK4(ODESolver):
    _kind = _capi.GOSS_RK4


class GRL1(ODESolver):
    _kind = _capi.GOSS_GRL1

    @staticmethod
    def default_parameters() -> Dict[str, Any]:
        names = ODESolver.default_parameters()
        names.update({"delta": 1e-8})
        return names


class GRL2(GRL1):
    _kind = _capi.GOSS_GRL2


class ImplicitODESolver(ODESolver, abc.ABC):
    @staticmethod
    def default_parameters() -> Dict[str, Any]:
        names = ODESolver.default_parameters()
        names.update({
            "eta_0": 1.0,
            "kappa": 0.1,
            "relative_tolerance": 1e-12,
            "max_iterations": 30,
            "max_relative_previous_residual": 0.01,
            "always_recompute_jacobian": False,
        })
        return names

    def num_jac_comp(self) -> int:
        """Number of Jacobian computations (summed over nodes for systems)."""
        return int(self._counters["jac_comp"])

    def compute_factorized_jacobian(self, y: np.ndarray, t: float, dt: float, alpha: float) -> None:
        """LU of (I - dt*alpha*J) (ImplicitODESolver.cpp:92-105); kept on the solver."""
        if self._ode is None:
            raise RuntimeError("no ODE attached to the solver")
        jac = self._ode.compute_jacobian(y, t)
        jac = np.ascontiguousarray(-dt * alpha * jac)
        jac[np.diag_indices_from(jac)] += 1.0
        self._ode.lu_factorize(jac)
        self._jac = jac
        self._counters["jac_comp"] += 1


class ImplicitEuler(ImplicitODESolver):
    _kind = _capi.GOSS_IMPLICIT_EULER

    @staticmethod
    def default_parameters() -> Dict[str, Any]:
        names = ImplicitODESolver.default_parameters()
        names.update({
            "num_refinements_without_always_recomputing_jacobian": 2,
            "min_dt": 0.0001,
        })
        return names


class ThetaSolver(ImplicitODESolver):
    _kind = _capi.GOSS_THETA

    @staticmethod
    def default_parameters() -> Dict[str, Any]:
        names = ImplicitODESolver.default_parameters()
        names.update({
            "num_refinements_without_always_recomputing_jacobian": 2,
            "min_dt": 0.0001,
            "theta": 0.5,
        })
        return names


class AdaptiveSolver(ODESolver, abc.ABC):
    _adaptive = True

    def __init__(self, *args, **kwargs):
        self._atol, self._rtol, self._iord = 1e-5, 1e-8, 3
        self._single_step = False
        super().__init__(*args, **kwargs)

    def get_current_time(self) -> float:
        return 0.0

    def get_current_time_step(self) -> float:
        return 0.0

    def get_num_accepted(self) -> int:
        return int(self._counters["accepted"])

    def get_num_rejected(self) -> int:
        return int(self._counters["rejected"])

    def set_single_step_mode(self, mode: bool) -> None:
        self._single_step = bool(mode)

    def set_tol(self, atol: float, rtol: float = 1e-8) -> None:
        self._atol, self._rtol = float(atol), float(rtol)

    def set_iord(self, iord: int) -> None:
        self._iord = int(iord)

    @property
    def atol(self):
        return self._atol

    @property
    def rtol(self):
        return self._rtol

    @property
    def iord(self) -> int:
        return self._iord


class AdaptiveImplicitSolver(ImplicitODESolver, AdaptiveSolver, abc.ABC):
    pass


class ESDIRK(AdaptiveImplicitSolver):
    @property
    def nfevals(self):
        """Number of right hand side evaluations"""
        return int(self._counters["nfevals"])

    @property
    def ndtsa(self):
        """Number of accepted timesteps"""
        return int(self._counters["ndtsa"])

    @property
    def ndtsr(self):
        """Number of rejected timesteps"""
        return int(self._counters["ndtsr"])


class ESDIRK23a(ESDIRK):
    _kind = _capi.GOSS_ESDIRK23A

    @staticmethod
    def default_parameters() -> Dict[str, Any]:
        names = AdaptiveImplicitSolver.default_parameters()
        names.update({
            "num_refinements_without_always_recomputing_jacobian": 2,
            "min_dt": 0.001,
        })
        return names


class GOSSSolvers(Enum):
    ExplicitEuler = "ExplicitEuler"
    RK2 = "RK2"
    RK4 = "RK4"
    RL1 = "RL1"
    RL2 = "RL2"
    GRL1 = "GRL1"
    GRL2 = "GRL2"
    ImplicitEuler = "ImplicitEuler"
    ThetaSolver = "ThetaSolver"
    ESDIRK23a = "ESDIRK23a"


class GOSSImplicitSolvers(Enum):
    ImplicitEuler = "ImplicitEuler"
    ThetaSolver = "ThetaSolver"
    ESDIRK23a = "ESDIRK23a"


class GOSSExplicitSolvers(Enum):
    ExplicitEuler = "ExplicitEuler"
    RK2 = "RK2"
    RK4 = "RK4"
    RL1 = "RL1"
    RL2 = "RL2"
    GRL1 = "GRL1"
    GRL2 = "GRL2"


class GOSSNonAdaptiveSolvers(Enum):
    ExplicitEuler = "ExplicitEuler"
    RK2 = "RK2"
    RK4 = "RK4"
    RL1 = "RL1"
    RL2 = "RL2"
    GRL1 = "GRL1"
    GRL2 = "GRL2"
    ImplicitEuler = "ImplicitEuler"
    ThetaSolver = "ThetaSolver"


class GOSSAdaptiveSolvers(Enum):
    ESDIRK23a = "ESDIRK23a"


solver_mapper = {
    "ExplicitEuler": ExplicitEuler,
    "RK2": RK2,
    "RK4": RK4,
    "RL1": RL1,
    "RL2": RL2,
    "GRL1": GRL1,
    "GRL2": GRL2,
    "ImplicitEuler": ImplicitEuler,
    "ThetaSolver": ThetaSolver,
    "ESDIRK23a": ESDIRK23a,
}
