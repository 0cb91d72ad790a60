"""The goss Python API on the GPU.

Ported from the reference tests ``tests/test_ode_bindings.py``,
``tests/test_ode_solver_bindings.py`` and
``tests/test_ode_system_solver_bindings.py``: known answers of the
oscillator, field state/parameter round trips, and every solver on a 4-node
oscillator system against cos/sin.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import goss_b200 as goss
from goss_b200._capi import GossError
from helpers import oracle_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oscilator():
    return goss.ParameterizedODE("oscilator")


def test_ode_eval(oscilator):
    assert np.allclose(oscilator.eval(np.array([0.1, 0.2]), 0), [-0.2, 0.1])
    assert np.allclose(oscilator.eval([0.1, 0.2], 0), [-0.2, 0.1])
    with pytest.raises(ValueError):
        oscilator.eval(np.array([0.1, 0.2, 0.3]), 0)


def test_ode_eval_component(oscilator):
    assert np.isclose(oscilator.eval_component(0, np.array([0.1, 0.2]), 0), -0.2)
    assert np.isclose(oscilator.eval_component(1, np.array([0.1, 0.2]), 0), 0.1)
    with pytest.raises(RuntimeError):
        oscilator.eval_component(3, np.array([0.1, 0.2]), 0)
    with pytest.raises(TypeError):
        oscilator.eval_component(-1, np.array([0.1, 0.2]), 0)


def test_ode_jacobian(oscilator):
    jac = oscilator.compute_jacobian(np.array([0.1, 0.2]), 0)
    assert np.allclose(jac, [[0, -1], [1, 0]])


@pytest.mark.parametrize("only_linear", [True, False])
def test_linearized_rhs(oscilator, only_linear):
    rhs, linear = oscilator.linearized_eval(np.array([0.1, 0.2]), 0, only_linear)
    if only_linear:
        assert linear is None
    else:
        assert np.allclose(linear, 0.0)
    assert np.allclose(rhs, [-0.2, 0.1])


def test_jacobian_and_lu_tt04_match_oracle():
    ode = goss.ParameterizedODE("tentusscher_2004_mcell")
    om = oracle_model("tentusscher_2004_mcell")
    ic = ode.get_ic()
    jac = ode.compute_jacobian(ic, 0.0)
    # forward differences with steps ~3e-8 |y| amplify last-bit differences of
    # the rhs (FMA contraction, libm vs CUDA exp) by ~1/delta
    ref = om.jacobian(ic, 0.0)
    assert np.allclose(jac, ref, rtol=1e-6, atol=1e-7 * np.abs(ref).max())
    ode.lu_factorize(jac)
    x = np.zeros_like(ic)
    ode.forward_backward_subst(jac, ic, x)
    assert np.isfinite(x).all()


def test_eval_matches_oracle_tp06():
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell")
    om = oracle_model("tentusscher_panfilov_2006_M_cell")
    rng = np.random.default_rng(2)
    ys = ode.get_ic()[None, :] * (1 + rng.uniform(-0.2, 0.2, (257, ode.num_states)))
    ts = rng.uniform(0, 20, 257)
    gpu = ode.eval_many(ys, ts)
    lin, rhs = ode.linearized_eval_many(ys, ts)
    cpu = np.array([om.rhs(y, t) for y, t in zip(ys, ts)])
    cl = np.array([om.linearized(y, t)[0] for y, t in zip(ys, ts)])
    # the device code folds parameter-only sub-expressions into constants,
    # which re-associates a few operations: agreement to rounding, amplified
    # only where terms of a sum cancel
    np.testing.assert_allclose(gpu, cpu, rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(rhs, cpu, rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(lin, cl, rtol=1e-11, atol=1e-14)


@pytest.mark.parametrize("Solver", goss.solvers.GOSSExplicitSolvers)
def test_solver_forward(Solver, oscilator):
    cls = goss.solvers.solver_mapper[Solver.name]
    y = oscilator.get_ic()
    solver = cls(oscilator)
    y_next = y.copy()
    solver.forward(y_next, 0, 0.1)
    assert np.allclose(y_next, [1, 0.1], rtol=0.01)


@pytest.mark.parametrize("Solver", goss.solvers.GOSSSolvers)
def test_solve_oscilator(Solver, oscilator):
    cls = goss.solvers.solver_mapper[Solver.name]
    solver = cls(oscilator)
    solver.internal_time_step = 0.0001
    dt = 0.1
    t = np.arange(0, 10.0 + dt, dt)
    u = solver.solve(t)
    assert np.isclose(u[:, 0], np.cos(t), rtol=0.14).all()
    assert np.isclose(u[:, 1], np.sin(t), rtol=0.02).all()


def test_construct_system(oscilator):
    solver = goss.solvers.ExplicitEuler()
    system = goss.ODESystemSolver(1, solver, oscilator)
    assert system.num_nodes == 1
    assert solver.get_ode().num_states == oscilator.num_states
    assert system.solver is solver and system.ode is oscilator
    assert system.num_threads == 0
    system.num_threads = 1
    assert system.num_threads == 1
    system.reset_default()


def test_states(oscilator):
    system = goss.ODESystemSolver(3, goss.solvers.ExplicitEuler(), oscilator)
    states = system.states
    assert states.shape == (3, 2)
    for node in range(3):
        assert np.allclose(states[node, :], oscilator.get_ic())


def test_field_states():
    ode = goss.ParameterizedODE("tentusscher_2004_mcell", field_states=["Ca_i", "V"],
                                field_parameters=["g_Kr", "g_Na", "g_Ks"])
    system = goss.ODESystemSolver(3, goss.solvers.ExplicitEuler(), ode)
    ic = ode.get_ic()
    vals = ic[ode.field_state_indices]
    fs = system.field_states
    assert fs.shape == (3, 2)
    assert (fs[:, 0] == vals[0]).all() and (fs[:, 1] == vals[1]).all()
    fs[:] = 0
    system.field_states = fs
    assert (system.field_states == 0).all()
    with pytest.raises(ValueError):
        system.field_states = np.zeros((4, 2))
    # into a caller's page-locked array
    pinned = torch.empty((3, 2), dtype=torch.float64, pin_memory=True).numpy()
    system.field_states = np.arange(6.0).reshape(3, 2)
    assert system.get_field_states(out=pinned) is pinned
    assert np.array_equal(pinned, np.arange(6.0).reshape(3, 2))


def test_field_state_components_untangled_layout():
    ode = goss.ParameterizedODE("tentusscher_2004_mcell", field_states=["Ca_i", "V"])
    system = goss.ODESystemSolver(5, goss.solvers.GRL1(ode), ode)
    system.set_field_state_components(np.arange(5.0), [1])
    v = system.get_field_state_components([1])[:, 0]
    assert np.array_equal(v, np.arange(5.0))
    assert np.array_equal(system.states[:, ode.state_names.index("V")], np.arange(5.0))
    # untangled (component-major) storage
    system._tangled_storage = False
    fs = system.field_states
    assert np.array_equal(fs.reshape(2, 5)[1], np.arange(5.0))


def test_field_parameters():
    ode = goss.ParameterizedODE("tentusscher_2004_mcell", field_states=["Ca_i", "V"],
                                field_parameters=["g_Kr", "g_Na", "g_Ks"])
    system = goss.ODESystemSolver(4, goss.solvers.ExplicitEuler(), ode)
    fp = system.field_parameters
    assert fp.shape == (4, 3)
    for i, name in enumerate(ode.field_parameter_names):
        assert np.allclose(fp[:, i], ode.parameters[name])
    fp[:] = 0
    system.field_parameters = fp
    assert (system.field_parameters == 0).all()


@pytest.mark.parametrize("Solver", goss.solvers.GOSSSolvers)
def test_solve_system_oscilator(Solver):
    cls = goss.solvers.solver_mapper[Solver.name]
    solver = cls()
    ode = goss.ParameterizedODE("oscilator", field_states=["x", "y"], field_parameters=["a", "b"])
    system = goss.ODESystemSolver(4, solver, ode)
    solver.internal_time_step = 0.0001
    dt = 0.1
    t = np.arange(0, 10.0 + dt, dt)
    fs = system.solve(t)
    for i in range(4):
        assert np.isclose(fs[:, i, 0], np.cos(t), rtol=0.14).all()
        assert np.isclose(fs[:, i, 1], np.sin(t), rtol=0.02).all()


def test_solve_equals_repeated_forward():
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell", field_states=["V", "Ca_i"])
    a = goss.ODESystemSolver(9, goss.solvers.GRL1(ode), ode)
    b = goss.ODESystemSolver(9, goss.solvers.GRL1(ode), ode)
    a.solver.internal_time_step = b.solver.internal_time_step = 0.01
    t = np.linspace(0, 20, 21)
    out = a.solve(t)
    for k in range(20):
        b.forward(t[k], t[k + 1] - t[k])
        assert np.array_equal(out[k + 1], b.field_states)


def test_model_parameter_change_after_construction():
    ode = goss.ParameterizedODE("oscilator")
    solver = goss.solvers.RK4(ode)
    system = goss.ODESystemSolver(2, solver, ode)
    ode.set_parameter("a", 0.0)
    ode.set_parameter("b", 0.0)
    system.forward(0.0, 1.0)
    assert np.allclose(system.states, ode.get_ic())


def test_monitored_values():
    ode = goss.ParameterizedODE("fitzhughnagumo", monitored=["p_42", "p_V"])
    ic = ode.get_ic()
    states = np.tile(ic, (3, 1))
    m = ode.monitored_values(states, np.arange(3.0))
    assert m.shape == (3, 2)
    assert np.allclose(m[:, 0], 42)
    assert np.allclose(m[:, 1], ic[0])
    assert np.allclose(ode.eval_monitored(ic, 0.0), [42.0, ic[0]])


def test_theta_newton_failure_raises():
    ode = goss.ParameterizedODE("tentusscher_2004_mcell")
    solver = goss.solvers.ThetaSolver(ode)
    solver.set_parameter("max_iterations", 0)
    solver.internal_time_step = 0.1
    system = goss.ODESystemSolver(3, solver, ode)
    with pytest.raises(RuntimeError, match="Newtons solver failed to converge as dt become smaller than 'min_dt'"):
        system.forward(0.0, 0.1)
    assert (system.node_status() & 2).all()


def test_nonfinite_states_flagged():
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell")
    system = goss.ODESystemSolver(4, goss.solvers.GRL1(ode), ode)
    y = system.states
    y[2, :] = np.nan
    system.set_states(y)
    system.forward(0.0, 0.1)
    assert system.status() & 1
    st = system.node_status()
    assert st[2] & 1 and not (st[[0, 1, 3]] & 1).any()
    system.status(clear=True)
    assert system.status() == 0


def test_fp32_precision_runs():
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell")
    system = goss.ODESystemSolver(64, goss.solvers.GRL1(ode), ode, precision="single")
    system.solver.internal_time_step = 0.01
    system.forward(0.0, 20.0)
    assert np.isfinite(system.states).all()
    with pytest.raises(GossError):
        goss.ODESystemSolver(4, goss.solvers.ThetaSolver(ode), ode, precision="single")


def test_measure_peaks_through_the_c_abi():
    """goss_measure_peaks (the roofline denominators of the model kernels):
    XU-pipe results and FP32 fused multiply-adds per second on cuda:0, in the
    range a B200-class GPU can give (nominal 4.65e12 and 3.72e13)."""
    import ctypes as C

    from goss_b200 import _capi

    xu, fp = C.c_double(0.0), C.c_double(0.0)
    assert _capi.lib().goss_measure_peaks(0, C.byref(xu), C.byref(fp)) == 0
    assert 1e12 < xu.value < 1e13, xu.value
    assert 1e13 < fp.value < 1e14, fp.value
    assert _capi.lib().goss_measure_peaks(0, None, C.byref(fp)) != 0  # NULL output rejected


def test_measure_fp64_peak_through_the_c_abi():
    """goss_measure_fp64_peak: FP64 fused multiply-adds per second on cuda:0
    (B200 nominal ~37 TFLOP/s FP64 vector, i.e. ~1.9e13 FMA/s)."""
    import ctypes as C

    from goss_b200 import _capi

    f = C.c_double(0.0)
    assert _capi.lib().goss_measure_fp64_peak(0, C.byref(f)) == 0
    assert 1e12 < f.value < 1e14, f.value
    assert _capi.lib().goss_measure_fp64_peak(0, None) != 0


def test_printed_fp64_grl1_matches_oracle():
    """GOSS_FP64_PRINTED: GRL1 with the model in its printed operation order
    (the plain FP64 path); within 1e-10 of the oracle like the split FP64."""
    import pyoracle
    from helpers import oracle_model, parity, perturbed_states

    N = 40
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell")
    om = oracle_model("tentusscher_panfilov_2006_M_cell")
    y0 = perturbed_states(om.ic, N, np.random.default_rng(4), 0.05)
    solver = goss.solvers.GRL1(ode)
    solver.internal_time_step = 0.01
    printed = goss.ODESystemSolver(N, solver, ode, precision="double_printed")
    assert printed.precision == "double_printed"
    printed.set_states(y0)
    o = pyoracle.OracleSystem(om, "GRL1", N, ldt=0.01)
    o.states[:] = y0
    for k in range(30):
        printed.forward(float(k), 1.0)
        o.forward(float(k), 1.0)
    assert parity(printed.states, o.states, rtol=1e-10) <= 1.0
    with pytest.raises(GossError):
        goss.ODESystemSolver(4, goss.solvers.RK4(ode), ode, precision="double_printed")


@pytest.mark.parametrize("tangled", [True, False])
def test_solve_matches_reference_solve(tangled):
    """goss_system_solve against the reference's own ODESystemSolver::solve
    (ODESystemSolver.cpp:81-99, oracle/_ref with a plugin whose field states
    are V and Ca_i): TP06 GRL1, 9 nodes, 21 output times over 20 ms,
    tangled and untangled storage, within 1e-10."""
    import ctypes as C

    import pyoracle
    from goss_b200 import _capi
    from helpers import meta, parity, perturbed_states, variant_dir

    name, fs = "tentusscher_panfilov_2006_M_cell", ("V", "Ca_i")
    plugin = pyoracle.field_state_plugin(name, fs) if pyoracle.ref_available() else None
    if plugin is None or not plugin.exists():
        pytest.skip("reference solvers (oracle/_ref) not built")
    om = oracle_model(name)
    N = 9
    y0 = perturbed_states(om.ic, N, np.random.default_rng(12), 0.05)
    t = np.linspace(0.0, 20.0, 21)
    r = pyoracle.RefSystem(plugin, meta(variant_dir(name))["class_name"], "GRL1", N, om.solver_params("GRL1", ldt=0.01))
    r.set_states(y0)
    ref = r.solve(t, tangled)
    ode = goss.ParameterizedODE(name, field_states=list(fs))
    system = goss.ODESystemSolver(N, goss.solvers.GRL1(ode), ode)
    system.solver.internal_time_step = 0.01
    system.set_states(y0)
    out = np.zeros_like(ref)
    system._sync_params()
    _capi.check(_capi.lib().goss_system_solve(system._h, out.ctypes.data_as(C.POINTER(C.c_double)),
                                              t.ctypes.data_as(C.POINTER(C.c_double)), t.size, int(tangled)),
                system._h)
    assert np.all(out[0] == 0.0) and np.all(ref[0] == 0.0)
    assert parity(out[1:], ref[1:], rtol=1e-10) <= 1.0
