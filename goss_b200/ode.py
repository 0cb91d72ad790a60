"""``ODE`` / ``ParameterizedODE``: the model objects of the goss Python API.

Mirrors ``goss.ode`` (reference ``python/goss/ode.py:40-231``): same
constructors, properties and methods.  A model is a compiled *variant*
(:mod:`goss_b200.compilemodule`); evaluations (``eval``, ``linearized_eval``,
``compute_jacobian``, ``eval_monitored``) run as batched CUDA kernels of that
variant.
"""
from __future__ import annotations

import os
from pathlib import Path
from typing import NamedTuple, Optional, Sequence

import numpy as np

from . import _capi
from .codegen.odeparse import ODEModel, ODEParseError
from .compilemodule import ModelModule, jit


class LinearizedEval(NamedTuple):
    rhs: np.ndarray
    linear: Optional[np.ndarray] = None


class _Bare:
    """Metadata-only model built from counts (``ParameterizedODE(num_states=3,
    num_parameters=1)`` in the reference, ``python/goss/ode.py:152-166``)."""

    def __init__(self, num_states, num_parameters, num_field_states=0, num_field_parameters=0, num_monitored=0):
        self.meta = dict(
            name="", state_names=[""] * num_states, parameter_names=[""] * num_parameters,
            field_parameter_names=[""] * num_field_parameters, field_parameter_indices=[0] * num_field_parameters,
            monitored_names=[""] * num_monitored, initial_conditions=[0.0] * num_states,
            default_parameters=[0.0] * num_parameters, linear_terms=[0] * num_states)
        self.num_field_states = num_field_states
        self.desc = None


class ODE:
    """A compiled model.

    ``ODE(path_or_model, field_states=[...], field_parameters=[...],
    monitored=[...])`` where the first argument is a ``.ode`` path, a parsed
    :class:`~goss_b200.codegen.odeparse.ODEModel`, the name of a shipped model,
    or another ``ODE``.
    """

    def __init__(self, *args, field_states: Sequence[str] = (), field_parameters: Sequence[str] = (),
                 monitored: Sequence[str] = (), linearization: str = "gotran", code_params: Optional[dict] = None,
                 **kwargs):
        if not args:
            raise ValueError("ODE needs a model")
        src = args[0]
        if isinstance(src, ODE):
            self._module = src._module
            self._params = src._params.copy()
            self._field_states = list(src._field_states)
            return
        if isinstance(src, (ODEModel, os.PathLike, str)):
            try:
                self._module = jit(src, field_parameters=field_parameters, monitored=monitored,
                                   linearization=linearization, code_params=code_params)
            except ODEParseError as exc:
                raise ValueError(str(exc)) from exc
            except ValueError:
                raise
        elif isinstance(src, ModelModule):
            self._module = src
        else:
            raise ValueError(f"Unknown argument of type {type(src)}")
        meta = self._module.meta
        for s in field_states:
            if s not in meta["state_names"]:
                raise ValueError(f"{s} is not a state in the {meta['name']} ODE")
        self._field_states = list(field_states)
        self._params = np.array(meta["default_parameters"], dtype=np.float64)

    # -- basic properties ---------------------------------------------------
    @property
    def _meta(self):
        return self._module.meta

    def __repr__(self) -> str:
        return f"{self.__class__.__name__}({self._meta['name']})"

    def __str__(self) -> str:
        return f"{self.__class__.__name__} with {self.num_states} states"

    def copy(self):
        return self.__class__(self)

    @property
    def name(self) -> str:
        return self._meta["name"]

    @property
    def num_states(self) -> int:
        return len(self._meta["state_names"])

    @property
    def is_dae(self) -> bool:
        return False

    def get_ic(self) -> np.ndarray:
        return np.array(self._meta["initial_conditions"], dtype=np.float64)

    @property
    def linear_terms(self) -> np.ndarray:
        return np.array(self._meta["linear_terms"], dtype=np.uint8)

    # -- evaluation (batched CUDA kernels) ------------------------------------
    def _check_state_input(self, states) -> np.ndarray:
        if len(states) != self.num_states:
            raise ValueError("State array has to be of same size as the number"
                             f"of states, got {len(states)}, expected {self.num_states}")
        return np.ascontiguousarray(states, dtype=np.float64)

    def _field_param_values(self) -> np.ndarray:
        idx = self._meta["field_parameter_indices"]
        return self._params[idx] if idx else np.zeros(0)

    def _eval(self, what: int, states: np.ndarray, times: np.ndarray, precision: int = _capi.GOSS_FP64,
              field_params: Optional[np.ndarray] = None) -> np.ndarray:
        states = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, self.num_states)
        count = states.shape[0]
        times = np.ascontiguousarray(np.broadcast_to(np.asarray(times, dtype=np.float64), (count,)))
        n = self.num_states
        width = {0: n, 1: 2 * n, 2: max(len(self._meta["monitored_names"]), 1), 3: n * n}[what]
        out = np.zeros((count, width))
        fp_ptr = None
        if field_params is not None:
            field_params = np.ascontiguousarray(field_params, dtype=np.float64).reshape(count, -1)
            fp_ptr = _capi.ptr(field_params)
        L = _capi.lib()
        _capi.check(L.goss_model_eval(self._module.desc, what, precision, _capi.ptr(self._params),
                                      _capi.ptr(states), fp_ptr, _capi.ptr(times), count, _capi.ptr(out), 0))
        return out

    def eval(self, states, time: float) -> np.ndarray:
        """Evaluate rhs of the ODE"""
        y = self._check_state_input(states)
        return self._eval(0, y, time)[0]

    def eval_many(self, states, times, precision: str = "double", field_params=None) -> np.ndarray:
        """Evaluate the rhs at many states at once ([count, n] -> [count, n])."""
        p = _capi.GOSS_FP32 if precision in ("single", "float", "float32", "fp32") else _capi.GOSS_FP64
        return self._eval(0, states, times, p, field_params)

    def linearized_eval_many(self, states, times, precision: str = "double", field_params=None):
        """(linear, rhs) at many states at once."""
        p = _capi.GOSS_FP32 if precision in ("single", "float", "float32", "fp32") else _capi.GOSS_FP64
        out = self._eval(1, states, times, p, field_params)
        n = self.num_states
        return out[:, :n], out[:, n:]

    def eval_component(self, component: int, states, time: float) -> float:
        """Evaluate component idx of the rhs of the ODE"""
        if not isinstance(component, (int, np.integer)) or isinstance(component, bool):
            raise TypeError("component must be an integer")
        if component < 0:
            raise TypeError("component must be a non-negative integer")
        if component >= self.num_states:
            raise RuntimeError("Index out of bounds")
        return float(self.eval(states, time)[component])

    def linearized_eval(self, states, time: float, only_linear: bool = False) -> LinearizedEval:
        """Evaluate the linearized rhs"""
        y = self._check_state_input(states)
        out = self._eval(1, y, time)[0]
        n = self.num_states
        linear, rhs = out[:n], out[n:]
        if only_linear:
            return LinearizedEval(rhs=rhs)
        return LinearizedEval(linear=linear, rhs=rhs)

    @property
    def has_jacobian(self) -> bool:
        """Generated with the analytic Jacobian (``code_params={"generate_jacobian": True}``)."""
        return bool(self._meta.get("jacobian", False))

    def compute_jacobian(self, states, time: float) -> np.ndarray:
        """Jacobian ``jac[i, j] = d f_i / d y_j``: the generated analytic one
        when the model has it (the reference's generated override), else
        forward differences (ODE::compute_jacobian, ODE.cpp:47-67) with the n+1
        right-hand sides evaluated in one batched kernel."""
        y = self._check_state_input(states)
        n = self.num_states
        if self.has_jacobian:
            return self._eval(3, y, time)[0].reshape(n, n)
        deltas = np.sqrt(1e-15 * np.maximum(1e-5, np.abs(y)))
        batch = np.repeat(y[None, :], n + 1, axis=0)
        batch[np.arange(1, n + 1), np.arange(n)] += deltas
        f = self._eval(0, batch, time)
        return np.ascontiguousarray((f[1:].T - f[0][:, None]) / deltas[None, :])

    def lu_factorize(self, mat: np.ndarray) -> None:
        """In place LU Factorize matrix (jacobian)"""
        if mat.dtype != np.float64 or not mat.flags.c_contiguous:
            raise TypeError("mat must be a C-contiguous float64 array")
        _capi.check(_capi.lib().goss_lu_factorize(mat.shape[0], _capi.ptr(mat)))

    def forward_backward_subst(self, mat: np.ndarray, b: np.ndarray, x: np.ndarray) -> None:
        """Forward/Backward substitution of factorized matrix"""
        mat = np.ascontiguousarray(mat, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise TypeError("x must be a C-contiguous float64 array")
        _capi.check(_capi.lib().goss_forward_backward_subst(mat.shape[0], _capi.ptr(mat), _capi.ptr(b),
                                                              _capi.ptr(x)))


class ParameterizedODE(ODE):
    """Model with named parameters, field states, field parameters and
    monitored intermediates (reference ``python/goss/ode.py:145-231``)."""

    def __init__(self, *args, **kwargs):
        if "num_states" in kwargs and "num_parameters" in kwargs:
            bare = _Bare(kwargs.get("num_states"), kwargs.get("num_parameters"), kwargs.get("num_field_states", 0),
                         kwargs.get("num_field_parameters", 0), kwargs.get("num_monitored", 0))
            self._module = bare
            self._field_states = [""] * bare.num_field_states
            self._params = np.zeros(kwargs.get("num_parameters"))
            return
        super().__init__(*args, **kwargs)

    @property
    def module(self) -> ModelModule:
        return self._module

    @property
    def num_parameters(self) -> int:
        return len(self._meta["parameter_names"])

    @property
    def num_field_parameters(self) -> int:
        return len(self._meta["field_parameter_names"])

    @property
    def num_field_states(self) -> int:
        return len(self._field_states)

    @property
    def num_monitored(self) -> int:
        return len(self._meta["monitored_names"])

    def eval_monitored(self, states, time: float) -> np.ndarray:
        if self.num_monitored == 0:
            raise RuntimeError(f"No monitored in the '{self.name.capitalize()}' model.")
        y = self._check_state_input(states)
        return self._monitored(y[None, :], np.array([float(time)]))[0]

    def monitored_values(self, states: np.ndarray, time: np.ndarray) -> np.ndarray:
        num_time_steps = len(time)
        assert states.shape == (num_time_steps, self.num_states)
        if self.num_monitored == 0:
            raise RuntimeError(f"No monitored in the '{self.name.capitalize()}' model.")
        return self._monitored(states, np.asarray(time, dtype=np.float64))

    def _monitored(self, states, times):
        out = self._eval(2, states, times)
        return out[:, : self.num_monitored]

    def set_parameter(self, name: str, value: float) -> None:
        try:
            i = self._meta["parameter_names"].index(name)
        except ValueError:
            raise RuntimeError(f'"{name}" is not a parameter in  this ODE.') from None
        self._params[i] = float(value)

    def get_parameter(self, name: str) -> float:
        try:
            i = self._meta["parameter_names"].index(name)
        except ValueError:
            raise RuntimeError(f'"{name}" is not a parameter in  this ODE.') from None
        return float(self._params[i])

    @property
    def parameter_values(self) -> np.ndarray:
        return self._params.copy()

    @property
    def parameters(self) -> dict:
        return {name: self.get_parameter(name) for name in self.parameter_names}

    @property
    def state_names(self) -> list:
        return list(self._meta["state_names"])

    @property
    def field_state_names(self) -> list:
        return list(self._field_states)

    @property
    def parameter_names(self) -> list:
        return list(self._meta["parameter_names"])

    @property
    def field_parameter_names(self) -> list:
        return list(self._meta["field_parameter_names"])

    @property
    def field_state_indices(self) -> list:
        names = self._meta["state_names"]
        return [names.index(s) for s in self._field_states]

    @property
    def monitored_names(self) -> list:
        return list(self._meta["monitored_names"])
