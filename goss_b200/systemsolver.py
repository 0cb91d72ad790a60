"""``ODESystemSolver``: one model at every node of a mesh, on the GPU.

Mirrors ``goss.ODESystemSolver`` (reference ``python/goss/systemsolver.py:15-134``
over ``cpp/goss/ODESystemSolver.{h,cpp}``) on top of the C ABI of
``include/goss_b200.h``.  Construction allocates the device state and applies
the initial conditions and default field parameters; ``forward`` advances
every node with the attached solver in one sm_100a kernel launch.

Solver and model parameters are read at every ``forward``/``solve`` (as the
reference reads the shared solver and ODE objects), so changing
``solver.internal_time_step`` or ``ode.set_parameter`` after construction
takes effect on the next step.

Extra keyword arguments beyond the reference API: ``precision`` ("double" —
FP64 everywhere —, "single": FP32 model arithmetic with FP64 state
accumulation, or "double_printed": FP64 with the model evaluated in the
printed operation order of the reference's generated code, GRL1 only) and
``device`` (CUDA ordinal).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _capi
from .ode import ParameterizedODE
from .solvers import ESDIRK, ImplicitODESolver, ODESolver


def has_shape(y: np.ndarray, xdim: int, ydim: int) -> bool:
    if y.shape == (xdim, ydim):
        return True
    if y.size == xdim * ydim:
        return True
    return False


def _precision(p) -> int:
    if p in (None, "double", "float64", "fp64", _capi.GOSS_FP64):
        return _capi.GOSS_FP64
    if p in ("single", "float", "float32", "fp32", _capi.GOSS_FP32):
        return _capi.GOSS_FP32
    if p in ("double_printed", _capi.GOSS_FP64_PRINTED):
        return _capi.GOSS_FP64_PRINTED
    raise ValueError(f"unknown precision {p!r}")


class ODESystemSolver:
    def __init__(self, num_nodes: int, solver: ODESolver, ode: ParameterizedODE, precision: str = "double",
                 device: int = 0):
        if not isinstance(solver, ODESolver):
            raise TypeError("solver must be a goss_b200.solvers.ODESolver")
        if getattr(ode, "_module", None) is None or getattr(ode._module, "desc", None) is None:
            raise TypeError("ode must be a compiled goss_b200.ParameterizedODE")
        if num_nodes < 0:
            raise ValueError("num_nodes must be non-negative")
        if solver.get_ode() is not ode:
            solver.attach(ode)
        self._solver = solver
        self._ode = ode
        self._tangled_storage = True
        self._precision = _precision(precision)
        self._device = int(device)
        self._L = _capi.lib()
        h = C.c_void_p()
        _capi.check(self._L.goss_system_create(ode._module.desc, solver.kind, solver.c_params(), int(num_nodes),
                                               self._precision, self._device, C.byref(h)))
        self._h = h
        self._num_nodes = int(num_nodes)
        fsi = np.array(ode.field_state_indices, dtype=np.uint32)
        _capi.check(self._L.goss_system_set_field_state_indices(
            self._h, fsi.ctypes.data_as(C.POINTER(C.c_uint32)), fsi.size), self._h)
        self._sync_params()
        # the constructor's reset_default uses the ODE's current parameters
        self.reset_default()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                self._L.goss_system_destroy(h)
            except Exception:
                pass
            self._h = None

    # -- parameter plumbing ---------------------------------------------------
    def _sync_params(self) -> None:
        _capi.check(self._L.goss_system_set_solver_params(self._h, self._solver.c_params()), self._h)
        for i, v in enumerate(self._ode._params):
            _capi.check(self._L.goss_system_set_parameter(self._h, i, float(v)), self._h)

    def _update_counters(self) -> None:
        if isinstance(self._solver, ImplicitODESolver):
            jc, rj, ac = self.counters()
            self._solver._counters["jac_comp"] = int(jc.sum())
            self._solver._counters["rejected"] = int(rj.sum())
            self._solver._counters["accepted"] = int(ac.sum())
            if isinstance(self._solver, ESDIRK):
                self._solver._counters["ndtsa"] = int(ac.sum())
                self._solver._counters["ndtsr"] = int(rj.sum())

    # -- reference API ---------------------------------------------------------
    @property
    def num_nodes(self) -> int:
        return self._num_nodes

    @property
    def solver(self) -> ODESolver:
        return self._solver

    @property
    def ode(self) -> ParameterizedODE:
        return self._ode

    @property
    def precision(self) -> str:
        return {_capi.GOSS_FP32: "single", _capi.GOSS_FP64_PRINTED: "double_printed"}.get(self._precision, "double")

    @property
    def num_threads(self) -> int:
        return int(self._L.goss_system_get_num_threads(self._h))

    @num_threads.setter
    def num_threads(self, num_threads: int) -> None:
        _capi.check(self._L.goss_system_set_num_threads(self._h, int(num_threads)), self._h)

    def reset_default(self) -> None:
        """Initial conditions and default field parameters at every node."""
        self._sync_params()
        _capi.check(self._L.goss_system_reset_default(self._h), self._h)

    @property
    def states(self) -> np.ndarray:
        """Copy of all states, shape (num_nodes, num_states)."""
        out = np.zeros((self._num_nodes, self._ode.num_states))
        _capi.check(self._L.goss_system_get_states(self._h, _capi.ptr(out)), self._h)
        return out

    def _set_states(self, states: np.ndarray) -> None:
        states = np.ascontiguousarray(states, dtype=np.float64)
        if not has_shape(states, self._num_nodes, self._ode.num_states):
            raise ValueError(f"Expected shape of states to be {(self._num_nodes, self._ode.num_states)}, "
                             f"got {states.shape}.")
        _capi.check(self._L.goss_system_set_states(self._h, _capi.ptr(states)), self._h)

    def set_states(self, states: np.ndarray) -> None:
        """Overwrite all states (the reference's mutable ``states()`` pointer)."""
        self._set_states(states)

    @property
    def field_parameters(self) -> np.ndarray:
        fp = np.zeros((self._num_nodes, self._ode.num_field_parameters))
        _capi.check(self._L.goss_system_get_field_parameters(self._h, _capi.ptr(fp), int(self._tangled_storage)),
                    self._h)
        return fp

    @field_parameters.setter
    def field_parameters(self, field_parameters: np.ndarray) -> None:
        field_parameters = np.ascontiguousarray(field_parameters, dtype=np.float64)
        if not has_shape(field_parameters, self._num_nodes, self._ode.num_field_parameters):
            raise ValueError(("Expected shape of field parameters to be "
                              f"{(self._num_nodes, self._ode.num_field_parameters)}, "
                              f"got {field_parameters.shape}."))
        _capi.check(self._L.goss_system_set_field_parameters(self._h, _capi.ptr(field_parameters),
                                                              int(self._tangled_storage)), self._h)

    @property
    def field_states(self) -> np.ndarray:
        fs = np.zeros((self._num_nodes, self._ode.num_field_states))
        _capi.check(self._L.goss_system_get_field_states(self._h, _capi.ptr(fs), int(self._tangled_storage)),
                    self._h)
        return fs

    @field_states.setter
    def field_states(self, field_states: np.ndarray) -> None:
        field_states = np.ascontiguousarray(field_states, dtype=np.float64)
        if not has_shape(field_states, self._num_nodes, self._ode.num_field_states):
            raise ValueError(("Expected shape of field states to be "
                              f"{(self._num_nodes, self._ode.num_field_states)}, "
                              f"got {field_states.shape}."))
        _capi.check(self._L.goss_system_set_field_states(self._h, _capi.ptr(field_states),
                                                          int(self._tangled_storage)), self._h)

    def get_field_states(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The field states, into ``out`` when given (a C-contiguous float64
        array of num_nodes x num_field_states values, e.g. in page-locked host
        memory the copy from the device can go to directly)."""
        if out is None:
            return self.field_states
        if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                and out.size == self._num_nodes * self._ode.num_field_states):
            raise ValueError("out must be a C-contiguous float64 array of "
                             f"{self._num_nodes * self._ode.num_field_states} values")
        _capi.check(self._L.goss_system_get_field_states(self._h, _capi.ptr(out), int(self._tangled_storage)),
                    self._h)
        return out

    def get_field_state_components(self, components) -> np.ndarray:
        comps = np.ascontiguousarray(components, dtype=np.uint32)
        out = np.zeros((self._num_nodes, self._ode.num_field_states))
        _capi.check(self._L.goss_system_get_field_state_components(
            self._h, _capi.ptr(out), comps.size, comps.ctypes.data_as(C.POINTER(C.c_uint32)),
            int(self._tangled_storage)), self._h)
        return out[:, comps]

    def set_field_state_components(self, values: np.ndarray, components) -> None:
        comps = np.ascontiguousarray(components, dtype=np.uint32)
        full = np.zeros((self._num_nodes, self._ode.num_field_states))
        full[:, comps] = np.asarray(values, dtype=np.float64).reshape(self._num_nodes, comps.size)
        _capi.check(self._L.goss_system_set_field_state_components(
            self._h, _capi.ptr(full), comps.size, comps.ctypes.data_as(C.POINTER(C.c_uint32)),
            int(self._tangled_storage)), self._h)

    def forward(self, t: float, interval: float) -> None:
        self._sync_params()
        _capi.check(self._L.goss_system_forward(self._h, float(t), float(interval)), self._h)
        self._update_counters()

    def solve(self, t: np.ndarray) -> np.ndarray:
        """Field states at every time of ``t``: shape (len(t), num_nodes, num_field_states)."""
        t = np.ascontiguousarray(t, dtype=np.float64)
        num_steps = t.size
        f0 = self.field_states
        field_states = np.zeros((num_steps, self._num_nodes, self._ode.num_field_states))
        field_states[0, :, :] = f0
        self._sync_params()
        _capi.check(self._L.goss_system_solve(self._h, _capi.ptr(field_states), _capi.ptr(t), num_steps,
                                              int(self._tangled_storage)), self._h)
        self._update_counters()
        return field_states

    # -- GPU extras ------------------------------------------------------------
    def forward_async(self, t: float, interval: float) -> None:
        """Enqueue a forward without waiting for it (parameters are not re-read)."""
        _capi.check(self._L.goss_system_forward_async(self._h, float(t), float(interval)), self._h)

    def synchronize(self) -> None:
        _capi.check(self._L.goss_system_synchronize(self._h), self._h)

    def capture(self, t0: float, interval: float, num_steps: int) -> None:
        """Record num_steps forward(t0 + k*interval, interval) launches into a
        CUDA graph (solver and model parameters as of now)."""
        self._sync_params()
        _capi.check(self._L.goss_system_capture(self._h, float(t0), float(interval), int(num_steps)), self._h)

    def replay(self) -> None:
        """Launch the captured graph and wait for it."""
        _capi.check(self._L.goss_system_replay(self._h), self._h)

    def set_block_size(self, block: int) -> None:
        _capi.check(self._L.goss_system_set_block_size(self._h, int(block)), self._h)

    def set_stream(self, stream_handle: int) -> None:
        _capi.check(self._L.goss_system_set_stream(self._h, C.c_void_p(stream_handle)), self._h)

    def status(self, clear: bool = False) -> int:
        f = C.c_uint32(0)
        _capi.check(self._L.goss_system_status(self._h, C.byref(f), int(clear)), self._h)
        return int(f.value)

    def node_status(self) -> np.ndarray:
        out = np.zeros(self._num_nodes, dtype=np.uint8)
        _capi.check(self._L.goss_system_node_status(self._h, out.ctypes.data_as(C.POINTER(C.c_uint8))), self._h)
        return out

    def counters(self):
        """Per-node (jacobian computations, rejected steps, accepted steps)."""
        jc = np.zeros(self._num_nodes, dtype=np.int64)
        rj = np.zeros(self._num_nodes, dtype=np.int64)
        ac = np.zeros(self._num_nodes, dtype=np.int64)
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))
        _capi.check(self._L.goss_system_counters(self._h, p(jc), p(rj), p(ac)), self._h)
        return jc, rj, ac

    def device_states(self):
        """(device pointer, leading dimension) of the FP64 state array [num_states][ld]."""
        ptr = C.POINTER(C.c_double)()
        ld = C.c_uint64(0)
        _capi.check(self._L.goss_system_device_states(self._h, C.byref(ptr), C.byref(ld)), self._h)
        return C.cast(ptr, C.c_void_p).value, int(ld.value)

    def device_field_params(self):
        ptr = C.POINTER(C.c_double)()
        ld = C.c_uint64(0)
        _capi.check(self._L.goss_system_device_field_params(self._h, C.byref(ptr), C.byref(ld)), self._h)
        return C.cast(ptr, C.c_void_p).value, int(ld.value)
