"""Heterogeneous batches (one persistent kernel for several populations),
CUDA-graph capture of forward loops, and the autotuner."""
from __future__ import annotations

import numpy as np
import pytest

import goss_b200 as goss
from goss_b200 import autotune
from helpers import parity

pytestmark = pytest.mark.gpu

F4 = ["g_Kr", "g_Ks", "g_CaL", "g_to"]
POPS = [  # model, field parameters, solver, nodes
    ("fitzhughnagumo", ["a", "b"], "RK4", 3),
    ("fitzhughnagumo", ["a", "b"], "RK4", 2000),
    ("oscilator", ["a", "b"], "RK4", 500),
    ("tentusscher_2004_mcell", F4, "GRL1", 700),
    ("tentusscher_panfilov_2006_M_cell", F4, "GRL1", 640),
    ("tentusscher_panfilov_2006_M_cell", F4, "GRL1", 1000),
]


def make_pops(precision="double", seed=4):
    rng = np.random.default_rng(seed)
    systems = []
    for model, fps, solver, n in POPS:
        ode = goss.ParameterizedODE(model, field_parameters=fps, field_states=[])
        s = goss.solvers.solver_mapper[solver](ode)
        s.internal_time_step = 0.01
        sysm = goss.ODESystemSolver(n, s, ode, precision=precision)
        y = ode.get_ic()[None, :] * (1 + rng.uniform(-0.1, 0.1, (n, ode.num_states)))
        fp = sysm.field_parameters * (1 + rng.uniform(-0.1, 0.1, (n, len(fps))))
        sysm.set_states(y)
        sysm.field_parameters = fp
        systems.append(sysm)
    return systems


def clone(systems):
    out = []
    for s in systems:
        solver = type(s.solver)(s.ode)
        solver.internal_time_step = s.solver.internal_time_step
        c = goss.ODESystemSolver(s.num_nodes, solver, s.ode, precision=s.precision)
        c.set_states(s.states)
        c.field_parameters = s.field_parameters
        out.append(c)
    return out


@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_matches_separate_systems(precision):
    pops = make_pops(precision)
    ref = clone(pops)
    batch = goss.BatchSolver(pops)
    for k in range(15):
        batch.forward(k * 0.5, 0.5)
        for r in ref:
            r.forward(k * 0.5, 0.5)
    # same per-node code in a different kernel: FP64 agrees to rounding; FP32
    # instruction selection may differ, so compare at FP32 accuracy
    tol = 1e-12 if precision == "double" else 1e-4
    for p, r in zip(pops, ref):
        assert np.isfinite(p.states).all()
        assert parity(p.states, r.states, rtol=tol, atol=1e-12) <= 1.0


@pytest.mark.parametrize("precision", ["double", "single"])
def test_schedules_and_orders_give_identical_results(precision):
    """Round-robin, atomic-counter and prefetching (rows staged in shared memory
    by bulk copies; populations of 3 and other odd-tile counts) schedules run
    the same arithmetic on the same values: bit-identical states."""
    results = []
    for cfg in (dict(block=128, grid=0, schedule=0), dict(block=64, grid=296, schedule=1, order=[5, 4, 3, 2, 1, 0]),
                dict(block=128, grid=148, schedule=0, order=[3, 1, 0, 2, 5, 4]),
                dict(block=64, grid=0, schedule=2), dict(block=128, grid=0, schedule=2, order=[3, 1, 0, 2, 5, 4]),
                dict(block=96, grid=7, schedule=2)):
        pops = make_pops(precision)
        batch = goss.BatchSolver(pops)
        batch.set_config(**cfg)
        for k in range(5):
            batch.forward(k * 1.0, 1.0)
        results.append([p.states for p in pops])
    for other in results[1:]:
        for a, b in zip(results[0], other):
            assert np.array_equal(a, b)


def test_batch_graph_replay_equals_forwards():
    a, b = make_pops(), make_pops()
    ba, bb = goss.BatchSolver(a), goss.BatchSolver(b)
    for k in range(10):
        ba.forward(k * 0.25, 0.25)
    bb.capture(0.0, 0.25, 10)
    bb.replay()
    for x, y in zip(a, b):
        assert np.array_equal(x.states, y.states)


@pytest.mark.parametrize("precision", ["double", "single"])
def test_fused_forwards_bit_identical_to_one_launch_per_forward(precision):
    """A captured graph runs its forwards all in one launch (the default),
    one per launch, or in ragged groups: the states stay on chip between the
    forwards of a launch (FP32 accumulators renormalised as a store and reload
    would), so every grouping gives the direct forwards' states bit for bit."""
    direct = make_pops(precision)
    bd = goss.BatchSolver(direct)
    for k in range(11):
        bd.forward(0.5 + k * 0.02, 0.02)
    for per, cfg in ((0, dict(block=128, grid=0, schedule=0)), (1, dict(block=64, grid=296, schedule=1)),
                     (3, dict(block=128, grid=0, schedule=2)), (4, dict(block=96, grid=7, schedule=1))):
        pops = make_pops(precision)
        b = goss.BatchSolver(pops)
        b.set_config(**cfg, forwards_per_launch=per)
        b.capture(0.5, 0.02, 11)
        b.replay()
        for x, y in zip(direct, pops):
            assert np.array_equal(x.states, y.states), (per, cfg)


def test_system_graph_replay_equals_forwards():
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell")
    s1 = goss.ODESystemSolver(300, goss.solvers.GRL1(ode), ode)
    s2 = goss.ODESystemSolver(300, goss.solvers.GRL1(ode), ode)
    s1.solver.internal_time_step = s2.solver.internal_time_step = 0.01
    for k in range(50):
        s1.forward(k * 0.01, 0.01)
    s2.capture(0.0, 0.01, 50)
    s2.replay()
    assert np.array_equal(s1.states, s2.states)


def test_autotuner_restores_states_and_applies_config():
    pops = make_pops()
    batch = goss.BatchSolver(pops)
    before = [p.states for p in pops]
    best = autotune.tune_batch(batch, interval=0.5, steps=2, use_cache=False,
                               candidates=[dict(block=128, grid=0, schedule=0, order=None),
                                           dict(block=64, grid=592, schedule=1, order=[5, 4, 3, 2, 1, 0])])
    assert best["tried"] == 2 and best["ms"] > 0
    assert batch.config["block"] == best["block"]
    for p, y in zip(pops, before):
        assert np.array_equal(p.states, y)


def test_batch_rejects_implicit_solvers():
    ode = goss.ParameterizedODE("tentusscher_2004_mcell")
    s = goss.ODESystemSolver(4, goss.solvers.ThetaSolver(ode), ode)
    with pytest.raises(ValueError):
        goss.BatchSolver([s])


def _oracle_pops(pops):
    """One oracle system (the C restatement of the reference solvers) per
    population, with the population's current states and field parameters."""
    import pyoracle
    from helpers import oracle_model

    out = []
    for (model, fps, solver, n), p in zip(POPS, pops):
        om = oracle_model(model, tuple(fps))
        o = pyoracle.OracleSystem(om, solver, n, ldt=0.01)
        o.states[:] = p.states
        o.field_params[:] = p.field_parameters
        out.append(o)
    return out


def test_batch_fp64_matches_oracle():
    """Every population of one persistent batch launch against the oracle
    directly: FP64 within 1e-10 (RK4 for FitzHugh-Nagumo and the oscillator,
    GRL1 for TT04 and TP06, per-node field parameters)."""
    pops = make_pops("double")
    oracles = _oracle_pops(pops)
    batch = goss.BatchSolver(pops)
    for k in range(15):
        batch.forward(k * 0.5, 0.5)
        for o in oracles:
            assert o.forward(k * 0.5, 0.5) == 0
    for p, o in zip(pops, oracles):
        assert parity(p.states, o.states, rtol=1e-10) <= 1.0


def test_batch_graph_fused_forwards_fp64_matches_oracle():
    """A captured graph of 40 forwards of 0.05 ms run in one launch (states on
    chip between forwards) against the oracle's 40 forward calls."""
    pops = make_pops("double", seed=6)
    oracles = _oracle_pops(pops)
    batch = goss.BatchSolver(pops)
    batch.capture(1.0, 0.05, 40)
    batch.replay()
    for k in range(40):
        for o in oracles:
            assert o.forward(1.0 + k * 0.05, 0.05) == 0
    for p, o in zip(pops, oracles):
        assert parity(p.states, o.states, rtol=1e-10) <= 1.0
