"""The FP64 tangent-linear checker (oracle/tangent) against the oracle.

The tangent-linear GRL1 trace is the reference against which the adjoint
kernels' gradients are checked, so it is pinned here first: its primal trace
equals the oracle's GRL1 trace (the reference's GRL1::forward), and its
Jacobian equals central finite differences of the oracle on a smooth model
to 1e-6.  On ten Tusscher-Panfilov, whose sodium-gate rates switch branches
discontinuously at V = -40 mV and whose upstroke amplifies rounding, central
differences agree only to ~1e-4 at their best step size; the tangent-linear
differentiates along the primal's branches without either error.
"""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from helpers import column_rel_err, meta, oracle_model, oracle_state_traces, parity, variant_dir


def _setup(name, fields, nodes, seed=3, spread=0.1):
    om = oracle_model(name, tuple(fields))
    vdir = variant_dir(name, fields)
    md = meta(vdir)
    rng = np.random.default_rng(seed)
    params = om.default_params
    idx = [md["parameter_names"].index(f) for f in fields]
    fp = params[idx][None, :] * np.exp(spread * rng.standard_normal((nodes, len(fields))))
    y0 = om.ic[None, :] * (1 + rng.uniform(-0.02, 0.02, (nodes, om.n)))
    return pyoracle.TangentTrace(vdir), om, md, params, fp, y0


def _fd(name, fields, fp, y0, interval, S, J, iv, dirs, n, h=1e-6):
    """Central differences of the oracle trace along each direction."""
    out = np.zeros((J, y0.shape[0], len(dirs)))
    for k, d in enumerate(dirs):
        yp, ym, fpp, fpm = y0.copy(), y0.copy(), fp.copy(), fp.copy()
        if d < n:
            step = h * np.maximum(np.abs(y0[:, d]), 1.0)
            yp[:, d] += step
            ym[:, d] -= step
        else:
            step = h * np.abs(fp[:, d - n])
            fpp[:, d - n] += step
            fpm[:, d - n] -= step
        tp = oracle_state_traces(name, fields, fpp, yp, interval, S, J, iv)
        tm = oracle_state_traces(name, fields, fpm, ym, interval, S, J, iv)
        out[:, :, k] = (tp - tm) / (2 * step[None, :])
    return out


def test_primal_trace_matches_oracle():
    name, fields = "tentusscher_panfilov_2006_M_cell", ["g_Kr", "g_Ks", "g_CaL", "g_to"]
    tl, om, md, params, fp, y0 = _setup(name, fields, 6)
    iv = md["state_names"].index("V")
    tr, jac = tl.trace(y0, fp, params, 0.0, 1.0, 100, 16, iv, [om.n + k for k in range(4)])
    ref = oracle_state_traces(name, fields, fp, y0, 1.0, 100, 16, iv)
    assert jac.shape == (16, 6, 4)
    assert parity(tr, ref, rtol=1e-10, atol=1e-12) <= 1.0


def test_jacobian_matches_central_differences_smooth_model():
    name, fields = "fitzhughnagumo", ["a", "b"]
    tl, om, md, params, fp, y0 = _setup(name, fields, 5)
    dirs = list(range(om.n + 2))   # both states and both fields
    S, J = 20, 30
    tr, jac = tl.trace(y0, fp, params, 0.0, 1.0, S, J, 0, dirs)
    # relative step 1e-4: truncation ~1e-8, rounding noise well below 1e-6
    fd = _fd(name, fields, fp, y0, 1.0, S, J, 0, dirs, om.n, h=1e-4)
    assert column_rel_err(jac.reshape(-1, len(dirs)), fd.reshape(-1, len(dirs))) < 1e-6


def test_jacobian_matches_central_differences_tp06_loosely():
    name, fields = "tentusscher_panfilov_2006_M_cell", ["g_Kr", "g_Ks", "g_CaL", "g_to"]
    tl, om, md, params, fp, y0 = _setup(name, fields, 4)
    iv = md["state_names"].index("V")
    dirs = [om.n + k for k in range(4)]
    tr, jac = tl.trace(y0, fp, params, 0.0, 1.0, 100, 16, iv, dirs)
    # rounding noise amplified through the upstroke dominates below h ~ 1e-4
    # (4e-3 at h = 1e-6 for g_Ks), branch switches above it
    fd = _fd(name, fields, fp, y0, 1.0, 100, 16, iv, dirs, om.n, h=1e-4)
    assert column_rel_err(jac.reshape(-1, 4), fd.reshape(-1, 4)) < 1e-3


def test_bad_arguments_raise():
    name, fields = "fitzhughnagumo", ["a", "b"]
    tl, om, md, params, fp, y0 = _setup(name, fields, 2)
    with pytest.raises(ValueError):
        tl.trace(y0, fp, params, 0.0, 1.0, 10, 2, 0, [om.n + 2])     # no such field
    with pytest.raises(ValueError):
        tl.trace(y0, fp, params, 0.0, 1.0, 10, 2, 0, list(range(33)) )


FIELD_VARIANTS = [("fitzhughnagumo", ["a", "b"]), ("oscilator", ["a", "b"]),
                  ("tentusscher_2004_mcell", ["g_Kr", "g_CaL"]),
                  ("tentusscher_2004_mcell", ["g_Kr", "g_Na", "g_Ks"]),
                  ("tentusscher_2004_mcell", ["g_Kr", "g_Ks", "g_CaL", "g_to"]),
                  ("tentusscher_panfilov_2006_M_cell", ["g_Kr", "g_Ks", "g_CaL", "g_to"])]


@pytest.mark.parametrize("name,fields", FIELD_VARIANTS, ids=lambda v: v if isinstance(v, str) else "-".join(v))
def test_generated_vjp_dot_product(name, fields):
    """The generated reverse sweep (linearized_vjp, compiled for the host in
    FP64) is the transpose of the forward-mode derivative of `linearized`:
    <abar, lin_dot> + <bbar, rhs_dot> = <ybar, ydot> + <Fbar, Fdot> for random
    directions and cotangents, at states on both sides of V = -40 mV."""
    tl, om, md, params, fp, y0 = _setup(name, fields, 6, seed=11)
    rng = np.random.default_rng(5)
    names = md["state_names"]
    worst = 0.0
    for node in range(6):
        y = y0[node].copy()
        if "V" in names:
            y[names.index("V")] = (-85.0, -60.0, -39.0, -20.0, 5.0, 30.0)[node]
        ydot = rng.standard_normal(om.n) * np.maximum(np.abs(y), 1e-3)
        Fdot = rng.standard_normal(len(fields)) * fp[node]
        abar, bbar = rng.standard_normal(om.n), rng.standard_normal(om.n)
        lin, rhs, lin_dot, rhs_dot = tl.jvp(y, fp[node], params, 12.5, ydot, Fdot)
        ybar, Fbar = tl.vjp(y, fp[node], params, 12.5, abar, bbar)
        lhs = abar @ lin_dot + bbar @ rhs_dot
        rhs_ = ybar @ ydot + Fbar @ Fdot
        scale = np.abs(abar * lin_dot).sum() + np.abs(bbar * rhs_dot).sum()
        worst = max(worst, abs(lhs - rhs_) / scale)
    assert worst < 1e-12, worst


def test_rk4_primal_and_jacobian_smooth_model():
    name, fields = "fitzhughnagumo", ["a", "b"]
    tl, om, md, params, fp, y0 = _setup(name, fields, 5)
    dirs = list(range(om.n + 2))
    S, J = 20, 30
    tr, jac = tl.trace(y0, fp, params, 0.0, 1.0, S, J, 0, dirs, solver="RK4")
    ref = oracle_state_traces(name, fields, fp, y0, 1.0, S, J, 0, solver="RK4")
    assert parity(tr, ref, rtol=1e-10, atol=1e-12) <= 1.0
    out = np.zeros_like(jac)
    h = 1e-4
    for k, d in enumerate(dirs):
        yp, ym, fpp, fpm = y0.copy(), y0.copy(), fp.copy(), fp.copy()
        if d < om.n:
            step = h * np.maximum(np.abs(y0[:, d]), 1.0)
            yp[:, d] += step
            ym[:, d] -= step
        else:
            step = h * np.abs(fp[:, d - om.n])
            fpp[:, d - om.n] += step
            fpm[:, d - om.n] -= step
        tp = oracle_state_traces(name, fields, fpp, yp, 1.0, S, J, 0, solver="RK4")
        tm = oracle_state_traces(name, fields, fpm, ym, 1.0, S, J, 0, solver="RK4")
        out[:, :, k] = (tp - tm) / (2 * step[None, :])
    assert column_rel_err(jac.reshape(-1, len(dirs)), out.reshape(-1, len(dirs))) < 1e-6
