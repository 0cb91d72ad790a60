"""Operator splitting with the PDE vector on the GPU (goss_b200.coupling).

A monodomain-like cable of 1,500 dofs: ten Tusscher-Panfilov M-cells on the
first 900 (node i at dof 899 - i, to exercise the dof maps), ten
Tusscher 2004 M-cells on the rest, V as the field state of both, GRL1 at
0.01 ms, and an explicit diffusion step in torch between ODE steps of 0.05 ms
(the stimulus at 10 ms starts the wave).  The device-resident coupling must
give the same V as the reference's way -- host copies of the field states
into and out of each population every step, diffusion in numpy -- to 1e-11,
and save/restore must return the populations to the saved states.
"""
from __future__ import annotations

import numpy as np
import pytest

import goss_b200 as goss
from goss_b200.coupling import FieldStateCoupling

pytestmark = pytest.mark.gpu

NUM_DOFS, DT, STEPS, D = 1500, 0.05, 240, 0.1   # D * DT / dx^2 with dx = 1


def populations():
    out = {}
    for label, model, n in (("tp06", "tentusscher_panfilov_2006_M_cell", 900),
                            ("tt04", "tentusscher_2004_mcell", NUM_DOFS - 900)):
        ode = goss.ParameterizedODE(model, field_states=["V"])
        s = goss.solvers.GRL1(ode)
        s.internal_time_step = 0.01
        out[label] = goss.ODESystemSolver(n, s, ode)
    # the first 900 dofs in reverse order for TP06, the rest for TT04
    dofs = {"tp06": np.arange(900)[::-1].copy(), "tt04": np.arange(900, NUM_DOFS)}
    return out, dofs


def diffuse_np(v):
    lap = np.empty_like(v)
    lap[1:-1] = v[:-2] - 2 * v[1:-1] + v[2:]
    lap[0] = v[1] - v[0]
    lap[-1] = v[-2] - v[-1]
    return v + D * lap


def diffuse_torch(v):
    import torch

    lap = torch.empty_like(v)
    lap[1:-1] = v[:-2] - 2 * v[1:-1] + v[2:]
    lap[0] = v[1] - v[0]
    lap[-1] = v[-2] - v[-1]
    v.add_(D * lap)


def initial_v(systems, dofs):
    v = np.zeros(NUM_DOFS)
    for lab, s in systems.items():
        v[dofs[lab]] = s.field_states[:, 0]
    return v


def test_device_coupling_matches_host_copies():
    import torch

    sys_h, dofs = populations()
    v = initial_v(sys_h, dofs)
    for k in range(STEPS):
        for lab, s in sys_h.items():          # to_field_states / forward / from_field_states
            s.field_states = v[dofs[lab]].reshape(-1, 1)
            s.forward(k * DT, DT)
            v[dofs[lab]] = s.field_states[:, 0]
        v = diffuse_np(v)

    sys_d, _ = populations()
    cpl = FieldStateCoupling(sys_d, dofs, NUM_DOFS)
    vd = torch.tensor(initial_v(sys_d, dofs), device="cuda")
    for k in range(STEPS):
        cpl.step((k * DT, (k + 1) * DT), vd)
        diffuse_torch(vd)
    cpl.synchronize()
    torch.cuda.synchronize()
    got = vd.cpu().numpy()
    assert np.isfinite(got).all() and got.max() > 0          # the wave is on its way
    assert np.max(np.abs(got - v) / np.maximum(np.abs(v), 1.0)) < 1e-11
    cpl.to_field_states(vd)                                   # the diffused V into the populations
    cpl.synchronize()
    for lab, s in sys_d.items():
        assert np.array_equal(s.field_states[:, 0], got[dofs[lab]])


def test_views_save_restore_and_errors():
    import torch

    systems, dofs = populations()
    cpl = FieldStateCoupling(systems, dofs, NUM_DOFS)
    views = cpl.field_state_views("tt04")
    assert len(views) == 1 and views[0].shape == (NUM_DOFS - 900,)
    before = {lab: s.states.copy() for lab, s in systems.items()}
    cpl.save_states()
    v = torch.full((NUM_DOFS,), -80.0, dtype=torch.float64, device="cuda")
    cpl.step((0.0, 1.0), v)
    cpl.synchronize()
    assert not np.array_equal(systems["tp06"].states, before["tp06"])
    cpl.restore_states()
    torch.cuda.synchronize()
    for lab, s in systems.items():
        assert np.array_equal(s.states, before[lab])
    with pytest.raises(TypeError):
        cpl.to_field_states(torch.zeros(NUM_DOFS, dtype=torch.float32, device="cuda"))
    with pytest.raises(ValueError):
        cpl.to_field_states(torch.zeros(NUM_DOFS + 1, dtype=torch.float64, device="cuda"))


def test_device_coupling_matches_reference_solvers():
    """The same cable with the reference's own solvers on the host arm: each
    population is the reference's compiled ODESystemSolver (oracle/_ref; the
    C restatement where it is not built) and V goes into and out of its field
    states every step, as DOLFINODESystemSolver.step does
    (python/goss/dolfinutils.py:750-780).  V within 1e-10 (of max(|V|, 1 mV))."""
    import torch

    import pyoracle
    from helpers import oracle_model, ref_system

    host = {}
    for label, model, n in (("tp06", "tentusscher_panfilov_2006_M_cell", 900),
                            ("tt04", "tentusscher_2004_mcell", NUM_DOFS - 900)):
        r = ref_system(model, "GRL1", n, ldt=0.01)
        if r is None:
            o = pyoracle.OracleSystem(oracle_model(model), "GRL1", n, ldt=0.01)
            r = (lambda o=o: o.states.copy(), lambda y, o=o: o.states.__setitem__(slice(None), y),
                 lambda t, dt, o=o: o.forward(t, dt))
        else:
            r = (r.get_states, r.set_states, r.forward)
        om = oracle_model(model)
        r[1](np.tile(om.ic, (n, 1)))
        host[label] = r
    sys_d, dofs = populations()
    iv = {lab: s.ode.state_names.index("V") for lab, s in sys_d.items()}
    v = initial_v(sys_d, dofs)
    v0 = v.copy()
    for k in range(STEPS):
        for lab, (get, put, fwd) in host.items():
            y = get()
            y[:, iv[lab]] = v[dofs[lab]]          # to_field_states
            put(y)
            assert fwd(k * DT, DT) == 0
            v[dofs[lab]] = get()[:, iv[lab]]       # from_field_states
        v = diffuse_np(v)

    cpl = FieldStateCoupling(sys_d, dofs, NUM_DOFS)
    vd = torch.tensor(v0, device="cuda")
    for k in range(STEPS):
        cpl.step((k * DT, (k + 1) * DT), vd)
        diffuse_torch(vd)
    cpl.synchronize()
    torch.cuda.synchronize()
    got = vd.cpu().numpy()
    assert got.max() > 0
    assert np.max(np.abs(got - v) / np.maximum(np.abs(v), 1.0)) < 1e-10
