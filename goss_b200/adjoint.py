"""Gradients of GRL1 and RK4 traces with respect to per-node field parameters.

``GRL1Trace`` / ``RK4Trace`` run the reference's user loop --
``forward(t0 + j*interval, interval)`` for ``j < num_intervals``, sampling
one state (``V`` by default) after every interval -- on the GPU and record a
checkpoint of the full state every ``checkpoint_every`` internal steps.  The
backward pass is a hand-written adjoint kernel
(``goss_b200/csrc/goss_adjoint.cuh``) that recomputes each checkpoint
segment and applies the transposed step Jacobians in reverse, using the
generated reverse-mode sweeps of the model's linearised right-hand side
(GRL1) or right-hand side (RK4).

:func:`trace` wraps it in a ``torch.autograd.Function``: any loss built from
the trace (for example a misfit ``((trace - target)**2).sum()``) can be
differentiated with respect to the field parameters and the initial states.
There is no counterpart in the reference, which has no gradients.
"""
from __future__ import annotations

import ctypes as C
import math
import numbers
from typing import Optional, Tuple

import numpy as np

from . import _capi
from .ode import ParameterizedODE

_AdjointFn = C.CFUNCTYPE(C.c_int, C.POINTER(_capi.AdjointLaunch))


def _ld(n: int) -> int:
    return (max(n, 1) + 31) // 32 * 32


class SolverTrace:
    """Trace of an explicit solve (GRL1 or RK4) over many nodes, with its adjoint.

    Parameters
    ----------
    ode : ParameterizedODE  (its field parameters are the differentiated inputs)
    num_nodes, interval (ms), steps_per_interval (internal steps per
    interval), num_intervals, checkpoint_every (internal steps; a multiple of
    steps_per_interval), trace_state (state name), precision ("single" or
    "double"), t0, device, solver ("GRL1" or "RK4").

    tape_bytes: device memory for a tape of every step's input state over the
    last checkpoint segments (0, the default: none; an int: at most that many
    bytes; ``"auto"``: the free device memory less ``tape_reserve`` bytes).
    The record pass writes the tape and the backward reads it instead of
    recomputing those segments from their checkpoints; the tape holds the
    values the recompute produces, so the gradient does not depend on it
    beyond rounding.  ``taped_segments`` reports how many segments fit.
    """

    SOLVERS = {"GRL1": _capi.GOSS_GRL1, "RK4": _capi.GOSS_RK4}

    def __init__(self, ode: ParameterizedODE, num_nodes: int, interval: float, steps_per_interval: int,
                 num_intervals: int, checkpoint_every: int, trace_state: str = "V", precision: str = "single",
                 t0: float = 0.0, device: int = 0, solver: str = "GRL1", tape_bytes=0,
                 tape_reserve: int = 2 << 30, reverse_precision: Optional[str] = None):
        import torch

        if solver not in self.SOLVERS:
            raise ValueError(f"no adjoint for solver {solver!r}; choose one of {sorted(self.SOLVERS)}")
        self.solver = solver
        if checkpoint_every % steps_per_interval:
            raise ValueError("checkpoint_every must be a multiple of steps_per_interval")
        if trace_state not in ode.state_names:
            raise ValueError(f"{trace_state} is not a state of {ode.name}")
        self.ode = ode
        self.N = int(num_nodes)
        self.n = ode.num_states
        self.nfp = ode.num_field_parameters
        self.interval = float(interval)
        self.S = int(steps_per_interval)
        self.J = int(num_intervals)
        self.K = int(checkpoint_every)
        self.t0 = float(t0)
        self.trace_index = ode.state_names.index(trace_state)
        self.precision = _capi.GOSS_FP32 if precision in ("single", "float32", "fp32") else _capi.GOSS_FP64
        # arithmetic of the backward's step VJPs: the trajectory's, or "double"
        # over an FP32 trajectory (GRL1)
        self.reverse_precision = self.precision if reverse_precision is None else (
            _capi.GOSS_FP32 if reverse_precision in ("single", "float32", "fp32") else _capi.GOSS_FP64)
        if self.reverse_precision != self.precision and not (
                self.precision == _capi.GOSS_FP32 and self.reverse_precision == _capi.GOSS_FP64 and solver == "GRL1"):
            raise ValueError("reverse_precision differs from precision only as FP64 over an FP32 GRL1 trajectory")
        self.device = torch.device("cuda", device)
        self.ld = _ld(self.N)
        total = self.J * self.S
        self.num_checkpoints = math.ceil(total / self.K)
        cp_dtype = torch.float32 if self.precision == _capi.GOSS_FP32 else torch.float64
        rows = 2 * self.n if self.precision == _capi.GOSS_FP32 else self.n
        dev = self.device
        self._checkpoints = torch.zeros((self.num_checkpoints, rows, self.ld), dtype=cp_dtype, device=dev)
        sld = (self.N + 255) // 256 * 256 + 256
        self._scratch = torch.zeros((self.K, self.n, sld), dtype=cp_dtype, device=dev)
        segment_bytes = self.K * self.n * sld * self._scratch.element_size()
        if tape_bytes == "auto":
            tape_bytes = torch.cuda.mem_get_info(dev)[0] - int(tape_reserve)
        elif not isinstance(tape_bytes, numbers.Integral) or isinstance(tape_bytes, bool):
            raise TypeError("tape_bytes must be an int or 'auto'")
        self.taped_segments = int(min(self.num_checkpoints, max(0, int(tape_bytes)) // segment_bytes))
        self._tape = (torch.empty((self.taped_segments, self.K, self.n, sld), dtype=cp_dtype, device=dev)
                      if self.taped_segments else None)
        self._states = torch.zeros((self.n, self.ld), dtype=torch.float64, device=dev)
        self._fp = torch.zeros((max(self.nfp, 1), self.ld), dtype=torch.float64, device=dev)
        self._trace = torch.zeros((self.J, self.ld), dtype=torch.float64, device=dev)
        self._flags = torch.zeros(1, dtype=torch.int32, device=dev)
        self._fn = _AdjointFn(ode.module.desc.contents.adjoint)
        if not ode.module.desc.contents.adjoint:
            raise _capi.ExtensionMissingError("the model module has no adjoint kernels")
        self.block = 0  # backward threads per block (0: chosen from the node count)
        self.final_states: Optional[object] = None

    def _launch(self, mode: int, trace_bar=None, fp_bar=None, states_bar=None) -> None:
        import torch

        L = _capi.AdjointLaunch()
        L.mode = mode
        L.solver = self.SOLVERS[self.solver]
        L.precision = self.precision
        L.num_nodes = self.N
        L.block = self.block
        L.ld = self.ld
        L.states = self._states.data_ptr()
        L.field_params = self._fp.data_ptr()
        params = np.ascontiguousarray(self.ode._params, dtype=np.float64)
        L.params = params.ctypes.data_as(C.POINTER(C.c_double))
        L.t0 = self.t0
        L.interval = self.interval
        L.num_intervals = self.J
        L.steps_per_interval = self.S
        L.checkpoint_every = self.K
        L.trace_state = self.trace_index
        L.checkpoints = self._checkpoints.data_ptr()
        L.trace = self._trace.data_ptr()
        L.trace_bar = trace_bar.data_ptr() if trace_bar is not None else None
        L.scratch = self._scratch.data_ptr()
        L.field_params_bar = fp_bar.data_ptr() if fp_bar is not None else None
        L.states_bar = states_bar.data_ptr() if states_bar is not None else None
        L.flags = self._flags.data_ptr()
        L.tape = self._tape.data_ptr() if self._tape is not None else None
        L.taped_segments = self.taped_segments
        L.reverse_precision = self.reverse_precision
        L.stream = torch.cuda.current_stream(self.device).cuda_stream
        rc = self._fn(C.byref(L))
        _capi.check(rc)

    def _to_rows(self, x, cols: int, out) -> None:
        """[N, cols] node-major tensor/array -> [cols][ld] device rows."""
        import torch

        t = torch.as_tensor(x, dtype=torch.float64, device=self.device).reshape(self.N, cols)
        out.zero_()
        out[:cols, : self.N] = t.t()

    def run_forward(self, field_params, states0=None):
        """Trace [num_intervals, N] (float64 tensor) from the given inputs."""
        import torch

        if states0 is None:
            states0 = torch.as_tensor(self.ode.get_ic(), device=self.device).expand(self.N, self.n)
        self._to_rows(states0, self.n, self._states)
        if self.nfp:
            self._to_rows(field_params, self.nfp, self._fp)
        self._launch(0)
        self.final_states = self._states[:, : self.N].t().clone()
        return self._trace[:, : self.N].clone()

    def run_backward(self, trace_bar) -> Tuple[object, object]:
        """(dL/dfield_params [N, nfp], dL/dstates0 [N, n]) from dL/dtrace."""
        import torch

        tb = torch.zeros((self.J, self.ld), dtype=torch.float64, device=self.device)
        tb[:, : self.N] = torch.as_tensor(trace_bar, dtype=torch.float64, device=self.device).reshape(self.J, self.N)
        fpb = torch.zeros((max(self.nfp, 1), self.ld), dtype=torch.float64, device=self.device)
        sb = torch.zeros((self.n, self.ld), dtype=torch.float64, device=self.device)
        self._launch(1, tb, fpb, sb)
        return fpb[: self.nfp, : self.N].t().clone(), sb[:, : self.N].t().clone()


class GRL1Trace(SolverTrace):
    """:class:`SolverTrace` of the GRL1 solver.  ``reverse_precision="double"``
    with ``precision="single"`` differentiates the FP32 trajectory with FP64
    step VJPs (separates the FP32 trajectory's share of the gradient error
    from the FP32 reverse arithmetic's)."""

    def __init__(self, ode: ParameterizedODE, num_nodes: int, interval: float, steps_per_interval: int,
                 num_intervals: int, checkpoint_every: int, trace_state: str = "V", precision: str = "single",
                 t0: float = 0.0, device: int = 0, tape_bytes=0, tape_reserve: int = 2 << 30,
                 reverse_precision: Optional[str] = None):
        super().__init__(ode, num_nodes, interval, steps_per_interval, num_intervals, checkpoint_every,
                         trace_state, precision, t0, device, solver="GRL1", tape_bytes=tape_bytes,
                         tape_reserve=tape_reserve, reverse_precision=reverse_precision)


class RK4Trace(SolverTrace):
    """:class:`SolverTrace` of the RK4 solver."""

    def __init__(self, ode: ParameterizedODE, num_nodes: int, interval: float, steps_per_interval: int,
                 num_intervals: int, checkpoint_every: int, trace_state: str = "V", precision: str = "single",
                 t0: float = 0.0, device: int = 0, tape_bytes=0, tape_reserve: int = 2 << 30):
        super().__init__(ode, num_nodes, interval, steps_per_interval, num_intervals, checkpoint_every,
                         trace_state, precision, t0, device, solver="RK4", tape_bytes=tape_bytes,
                         tape_reserve=tape_reserve)


def _function():
    import torch

    class _TraceFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, field_params, states0, solver: SolverTrace):
            ctx.solver = solver
            return solver.run_forward(field_params.detach(), states0.detach())

        @staticmethod
        def backward(ctx, grad_trace):
            gfp, gy0 = ctx.solver.run_backward(grad_trace.contiguous())
            return gfp, gy0, None

    return _TraceFn


_TRACE_FN = None


def trace(solver: SolverTrace, field_params, states0=None):
    """Differentiable trace: ``solver``'s GRL1 loop as a torch function of the
    field parameters [N, nfp] and the initial states [N, n]."""
    import torch

    global _TRACE_FN
    if _TRACE_FN is None:
        _TRACE_FN = _function()
    if states0 is None:
        states0 = torch.as_tensor(solver.ode.get_ic(), dtype=torch.float64,
                                  device=solver.device).expand(solver.N, solver.n).contiguous()
    return _TRACE_FN.apply(field_params, states0, solver)
