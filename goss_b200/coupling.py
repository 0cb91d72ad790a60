"""Operator-splitting exchange between a PDE vector on the GPU and the field
states of one or more ODE populations.

In goss the caller of this path is ``DOLFINODESystemSolver``
(``python/goss/dolfinutils.py:670-780``): every PDE time step it copies the
PDE unknowns (e.g. the membrane potential V at the mesh vertices) into the
field states of each cell population's ``ODESystemSolver``
(``to_field_states``), advances the ODEs (``forward``) and copies the field
states back (``from_field_states``) -- host copies of the whole vector on
every step.  :class:`FieldStateCoupling` does the same with the PDE vector as
a CUDA ``torch`` tensor: the field states are read and written in place
through zero-copy views of the solvers' device state rows, and the copies,
the ODE launches and the caller's PDE kernels are ordered on one CUDA stream,
so nothing crosses PCIe between steps.

``dofs[label]`` plays the role of the reference's dof maps: entry ``i`` is
the PDE dof of node ``i`` of that population.  A PDE vector holds one field
(shape ``(num_dofs,)``) or several (``(num_dofs, num_fields)``, the field
states of every population in the same order).
"""
from __future__ import annotations

from typing import Dict, Mapping, Optional, Tuple

import numpy as np

from .systemsolver import ODESystemSolver


def check_dof_maps(num_dofs: int, maps: Mapping[str, Tuple[int, np.ndarray]]) -> None:
    """Validate dof maps {label: (num_nodes, dofs)}: one entry per node, every
    dof in [0, num_dofs), no dof owned by two nodes.  Raises ValueError."""
    owner = np.full(num_dofs, -1, dtype=np.int64)
    for k, (label, (num_nodes, dofs)) in enumerate(maps.items()):
        d = np.asarray(dofs)
        if d.ndim != 1 or d.size != num_nodes:
            raise ValueError(f"dofs[{label!r}] must have one entry per node ({num_nodes}), got shape {d.shape}")
        if not np.issubdtype(d.dtype, np.integer):
            raise ValueError(f"dofs[{label!r}] must be integers")
        if d.size and (d.min() < 0 or d.max() >= num_dofs):
            raise ValueError(f"dofs[{label!r}] has entries outside [0, {num_dofs})")
        if np.unique(d).size != d.size:
            raise ValueError(f"dofs[{label!r}] maps two nodes to one dof")
        taken = owner[d] >= 0
        if taken.any():
            raise ValueError(f"dofs[{label!r}] overlaps another population at dof {int(d[taken][0])}")
        owner[d] = k


class _CudaArray:
    """__cuda_array_interface__ of one row of a solver's device state array."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


class FieldStateCoupling:
    """Device-resident ``to_field_states`` / ``step`` / ``from_field_states``.

    Parameters
    ----------
    systems : {label: ODESystemSolver}, all on one device, each with the same
        number of field states
    dofs : {label: int array}, the PDE dof of every node of that population
    num_dofs : length of the PDE vector
    """

    def __init__(self, systems: Mapping[str, ODESystemSolver], dofs: Mapping[str, object], num_dofs: int):
        import torch

        if not systems:
            raise ValueError("at least one ODESystemSolver is needed")
        if set(systems) != set(dofs):
            raise ValueError("systems and dofs must have the same labels")
        nfs = {s.ode.num_field_states for s in systems.values()}
        if len(nfs) != 1 or 0 in nfs:
            raise ValueError("every population needs the same, non-zero number of field states")
        self.num_fields = nfs.pop()
        self.num_dofs = int(num_dofs)
        dof_np = {lab: np.asarray(d.cpu() if hasattr(d, "cpu") else d) for lab, d in dofs.items()}
        check_dof_maps(self.num_dofs, {lab: (systems[lab].num_nodes, dof_np[lab]) for lab in systems})
        devices = {s._device for s in systems.values()}
        if len(devices) != 1:
            raise ValueError("all populations must live on one device")
        self.device = torch.device("cuda", devices.pop())
        self.systems: Dict[str, ODESystemSolver] = dict(systems)
        self.dofs = {lab: torch.as_tensor(dof_np[lab], dtype=torch.int64, device=self.device) for lab in systems}
        self._views = {}
        for lab, s in self.systems.items():
            ptr, ld = s.device_states()
            rows = s.ode.field_state_indices
            self._views[lab] = [torch.as_tensor(_CudaArray(ptr + 8 * ld * int(r), s.num_nodes), device=self.device)
                                for r in rows]
        self._saved: Optional[Dict[str, object]] = None
        self.use_stream(torch.cuda.current_stream(self.device))

    def use_stream(self, stream) -> None:
        """Run the ODE launches on ``stream`` (a torch.cuda.Stream), the stream
        the caller's PDE work and this object's copies run on."""
        self.stream = stream
        for s in self.systems.values():
            s.set_stream(stream.cuda_stream)

    def field_state_views(self, label: str):
        """Zero-copy float64 CUDA tensors, one per field state, of the nodes of
        population ``label`` (node order); valid while that solver lives."""
        return list(self._views[label])

    def _vector(self, v):
        import torch

        if not (isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float64):
            raise TypeError("the PDE vector must be a float64 CUDA tensor")
        if v.shape[0] != self.num_dofs or (v.dim() == 2 and v.shape[1] != self.num_fields) or v.dim() > 2 or \
                (v.dim() == 1 and self.num_fields != 1):
            raise ValueError(f"PDE vector of shape {tuple(v.shape)}; expected ({self.num_dofs},"
                             f"{'' if self.num_fields == 1 else ' ' + str(self.num_fields)})")
        return v if v.dim() == 2 else v.view(-1, 1)

    def to_field_states(self, v) -> None:
        """Copy the PDE vector into the populations' field states
        (``DOLFINODESystemSolver.to_field_states``)."""
        import torch

        v2 = self._vector(v)
        with torch.cuda.stream(self.stream):
            for lab, views in self._views.items():
                vals = v2.index_select(0, self.dofs[lab])
                for k, view in enumerate(views):
                    view.copy_(vals[:, k])

    def from_field_states(self, v) -> None:
        """Copy the populations' field states into the PDE vector
        (``DOLFINODESystemSolver.from_field_states``)."""
        import torch

        v2 = self._vector(v)
        with torch.cuda.stream(self.stream):
            for lab, views in self._views.items():
                vals = torch.stack(views, dim=1)
                v2.index_copy_(0, self.dofs[lab], vals)

    def update_parameters(self) -> None:
        """Push solver and model parameters changed on the host to every
        population (``DOLFINODESystemSolver.update_parameters``)."""
        for s in self.systems.values():
            s._sync_params()

    def step(self, interval: Tuple[float, float], v) -> None:
        """One ODE step of the splitting on (t0, t1): to_field_states, forward
        of every population, from_field_states (``DOLFINODESystemSolver.step``),
        all enqueued on the coupling's stream without waiting."""
        t0, t1 = interval
        self.to_field_states(v)
        for s in self.systems.values():
            s.forward_async(float(t0), float(t1) - float(t0))
        self.from_field_states(v)

    def synchronize(self) -> None:
        """Wait for everything enqueued so far and raise on a node failure."""
        for s in self.systems.values():
            s.synchronize()

    def save_states(self) -> None:
        """Keep a device copy of every population's full state
        (``DOLFINODESystemSolver.save_states``)."""
        import torch

        saved = {}
        with torch.cuda.stream(self.stream):
            for lab, s in self.systems.items():
                ptr, ld = s.device_states()
                rows = [torch.as_tensor(_CudaArray(ptr + 8 * ld * i, s.num_nodes), device=self.device)
                        for i in range(s.ode.num_states)]
                saved[lab] = (rows, torch.stack(rows).clone())
        self._saved = saved

    def restore_states(self) -> None:
        """Put back the states kept by :meth:`save_states`
        (``DOLFINODESystemSolver.restore_states``)."""
        import torch

        if self._saved is None:
            raise RuntimeError("no saved states")
        with torch.cuda.stream(self.stream):
            for lab, (rows, copy) in self._saved.items():
                for i, row in enumerate(rows):
                    row.copy_(copy[i])
