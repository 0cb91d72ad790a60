"""The oracle itself: the C restatement against the reference's own solvers.

``oracle/_ref`` is the reference's ``cpp/goss`` solvers compiled directly
from its sources; the restatement must reproduce them bit for bit (same
arithmetic, same order, same compiler flags).  Skipped when ``oracle/_ref``
was not built (no reference sources on this machine).
"""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from helpers import meta, oracle_model, perturbed_states, ref_system, variant_dir

pytestmark = pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref not built")

CASES = [
    # model, solver, nodes, steps, interval, internal step
    ("tentusscher_panfilov_2006_M_cell", "GRL1", 8, 1500, 0.01, 0.01),
    ("tentusscher_panfilov_2006_M_cell", "GRL2", 8, 150, 0.1, 0.1),
    ("tentusscher_panfilov_2006_M_cell", "RK4", 8, 1500, 0.01, 0.005),
    ("tentusscher_panfilov_2006_M_cell", "ExplicitEuler", 8, 1500, 0.01, 0.001),
    ("tentusscher_2004_mcell", "ThetaSolver", 4, 150, 0.1, 0.1),
    ("tentusscher_2004_mcell", "ESDIRK23a", 4, 60, 0.1, -1.0),
    ("beeler_reuter_1977", "GRL1", 8, 1500, 0.01, 0.01),
    ("fitzhughnagumo", "RK4", 8, 500, 0.1, 0.01),
    ("tentusscher_panfilov_2006_M_cell", "RL1", 8, 1500, 0.01, 0.01),
    ("tentusscher_panfilov_2006_M_cell", "RL2", 8, 150, 0.1, 0.1),
    ("tentusscher_panfilov_2006_M_cell", "RK2", 8, 1500, 0.01, 0.005),
    ("beeler_reuter_1977", "RL2", 8, 1500, 0.01, 0.01),
    ("fitzhughnagumo", "RK2", 8, 500, 0.1, 0.01),
    ("tentusscher_2004_mcell", "ImplicitEuler", 4, 150, 0.1, 0.1),
    ("tentusscher_2004_mcell", "ImplicitEuler", 4, 60, 0.1, -1.0),
]


@pytest.mark.parametrize("model,solver,N,steps,dt,ldt", CASES)
def test_restatement_bit_identical_to_reference(model, solver, N, steps, dt, ldt):
    rng = np.random.default_rng(7)
    om = oracle_model(model)
    y0 = perturbed_states(om.ic, N, rng, spread=0.02)
    o = pyoracle.OracleSystem(om, solver, N, ldt=ldt)
    o.states[:] = y0
    r = ref_system(model, solver, N, ldt=ldt)
    if r is None:
        pytest.skip("reference plugin not built")
    r.set_states(y0)
    for k in range(steps):
        assert o.forward(k * dt, dt, threads=4) == 0
        assert r.forward(k * dt, dt) == 0
    a, b = o.states.copy(), r.get_states()
    assert np.array_equal(a, b, equal_nan=True), float(np.nanmax(np.abs(a - b)))
    if solver in ("ThetaSolver", "ESDIRK23a", "ImplicitEuler"):
        jc, _, _ = o.counters()
        assert np.array_equal(jc, r.num_jac_comp())


def test_restatement_field_parameters_match_reference():
    name, fps = "tentusscher_panfilov_2006_M_cell", ("g_Kr", "g_Ks", "g_CaL", "g_to")
    rng = np.random.default_rng(3)
    om = oracle_model(name, fps)
    N = 6
    defaults = om.default_params[[meta(variant_dir(name, fps))["parameter_names"].index(p) for p in fps]]
    fp = defaults[None, :] * np.exp(0.2 * rng.standard_normal((N, len(fps))))
    o = pyoracle.OracleSystem(om, "GRL1", N, ldt=0.01)
    o.field_params[:] = fp
    r = ref_system(name, "GRL1", N, field_parameters=fps, ldt=0.01)
    if r is None:
        pytest.skip("reference plugin not built")
    r.set_field_parameters(fp)
    for k in range(1500):
        o.forward(k * 0.01, 0.01, threads=2)
        r.forward(k * 0.01, 0.01)
    assert np.array_equal(o.states, r.get_states())


def test_theta_newton_failure_reported_by_both():
    """max_iterations=0 makes every Newton solve fail: the step is halved
    until it falls below min_dt and the reference throws."""
    om = oracle_model("tentusscher_2004_mcell")
    o = pyoracle.OracleSystem(om, "ThetaSolver", 2, ldt=0.1, max_iterations=0)
    assert o.forward(0.0, 0.1) == 2
    r = ref_system("tentusscher_2004_mcell", "ThetaSolver", 2, ldt=0.1, max_iterations=0)
    if r is None:
        pytest.skip("reference plugin not built")
    assert r.forward(0.0, 0.1) == 2
