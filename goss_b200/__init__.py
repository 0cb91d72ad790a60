"""goss_b200: goss's multi-node ODE solve path on NVIDIA B200 (sm_100a).

Drop-in for the ``goss`` Python entry points of that path
(reference ``python/goss/__init__.py``):

* :class:`ParameterizedODE` / :class:`ODE` -- compiled cell models from
  gotran ``.ode`` files (own parser and code generator, CUDA device code)
* :mod:`solvers` -- ExplicitEuler, RK2, RK4, RL1, RL2, GRL1, GRL2,
  ImplicitEuler, ThetaSolver, ESDIRK23a
* :class:`ODESystemSolver` -- one model at every mesh node on the GPU
* :class:`FieldStateCoupling` -- operator-splitting exchange with a PDE
  vector kept on the GPU (the role of ``DOLFINODESystemSolver``)

The compute path is the CUDA runtime ``goss_b200/_lib/libgoss_b200.so`` and
one ``libgoss_model.so`` per model variant; there is no CPU fallback.
"""
from __future__ import annotations

from . import codegen, solvers
from .codegen.odeparse import ODEModel, load_ode
from .compilemodule import jit
from .ode import ODE, LinearizedEval, ParameterizedODE
from .systemsolver import ODESystemSolver

__version__ = "0.1.0"


def has_openmp() -> bool:
    """Whether nodes are solved in parallel.

    The reference reports its OpenMP build flag here
    (``cpp/goss/ODESystemSolver.cpp:7-13``); every node of a goss_b200 system
    runs in parallel on the GPU, so this is always True.
    """
    return True


__all__ = [
    "codegen",
    "jit",
    "load_ode",
    "ODE",
    "ODEModel",
    "solvers",
    "ODESystemSolver",
    "ParameterizedODE",
    "LinearizedEval",
    "has_openmp",
    "__version__",
]

from .batch import BatchSolver  # noqa: E402
from .coupling import FieldStateCoupling  # noqa: E402

__all__ += ["BatchSolver", "FieldStateCoupling"]
