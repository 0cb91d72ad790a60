"""Adjoint of GRL1 traces (goss_b200.adjoint) against finite differences.

The trace is the reference's user loop (forward(t0 + j*interval, interval),
V sampled after each interval); the loss a trace misfit.  Checks:

* the FP64 record kernel reproduces the oracle's trace (the reference's
  GRL1 semantics) to 1e-10;
* FP64 adjoint gradients w.r.t. the four conductance fields equal central
  finite differences (relative step 1e-6) of the ORACLE's FP64 loss;
* the same against GPU FP64 central differences on every node;
* checkpoint spacing does not change the gradient;
* the FP32 adjoint against the FP64 adjoint.
"""
from __future__ import annotations

import numpy as np
import pytest

import goss_b200 as goss
import pyoracle
from goss_b200.adjoint import GRL1Trace, trace
from helpers import oracle_model, parity

pytestmark = pytest.mark.gpu

F4 = ["g_Kr", "g_Ks", "g_CaL", "g_to"]
MODEL = "tentusscher_panfilov_2006_M_cell"
N, S, J, INTERVAL = 24, 100, 16, 1.0   # 16 ms with the stimulus at 10 ms


def setup(precision="double", K=400, seed=2):
    import torch

    ode = goss.ParameterizedODE(MODEL, field_parameters=F4)
    rng = np.random.default_rng(seed)
    defaults = np.array([ode.get_parameter(p) for p in F4])
    fp = defaults[None, :] * np.exp(0.2 * rng.standard_normal((N, 4)))
    fp_target = defaults[None, :] * np.exp(0.2 * rng.standard_normal((N, 4)))
    y0 = ode.get_ic()[None, :] * (1 + rng.uniform(-0.02, 0.02, (N, ode.num_states)))
    tr = GRL1Trace(ode, N, INTERVAL, S, J, K, precision=precision)
    target = tr.run_forward(torch.tensor(fp_target, device="cuda"), torch.tensor(y0, device="cuda")).clone()
    return ode, tr, fp, y0, target


def loss_grad(tr, fp, y0, target):
    import torch

    p = torch.tensor(fp, device="cuda", requires_grad=True)
    v = trace(tr, p, torch.tensor(y0, device="cuda"))
    loss = ((v - target) ** 2).sum()
    loss.backward()
    return float(loss), p.grad.cpu().numpy(), v.detach().cpu().numpy()


def oracle_traces(ode, fp, y0):
    """Oracle (reference semantics) traces of V for every row of fp."""
    om = oracle_model(MODEL, tuple(F4))
    n_sys = fp.shape[0]
    o = pyoracle.OracleSystem(om, "GRL1", n_sys, ldt=INTERVAL / S)
    o.states[:] = y0
    o.field_params[:] = fp
    iv = ode.state_names.index("V")
    out = np.zeros((J, n_sys))
    for j in range(J):
        o.forward(j * INTERVAL, INTERVAL)
        out[j] = o.states[:, iv]
    return out


def test_record_trace_matches_oracle():
    import torch

    ode, tr, fp, y0, target = setup()
    v = tr.run_forward(torch.tensor(fp, device="cuda"), torch.tensor(y0, device="cuda")).cpu().numpy()
    ref = oracle_traces(ode, fp, y0)
    assert parity(v, ref, rtol=1e-10, atol=1e-12) <= 1.0


def test_adjoint_matches_oracle_central_differences():
    ode, tr, fp, y0, target = setup()
    _, grad, _ = loss_grad(tr, fp, y0, target)
    tgt = target.cpu().numpy()
    nodes = [0, 5, 11, 23]
    h = 1e-6
    for k in range(4):
        fpp, fpm = fp[nodes].copy(), fp[nodes].copy()
        fpp[:, k] *= 1 + h
        fpm[:, k] *= 1 - h
        lp = ((oracle_traces(ode, fpp, y0[nodes]) - tgt[:, nodes]) ** 2).sum(axis=0)
        lm = ((oracle_traces(ode, fpm, y0[nodes]) - tgt[:, nodes]) ** 2).sum(axis=0)
        fd = (lp - lm) / (2 * h * fp[nodes, k])
        np.testing.assert_allclose(grad[nodes, k], fd, rtol=2e-5, atol=1e-9 * np.abs(fd).max())


def test_adjoint_matches_gpu_central_differences_all_nodes():
    import torch

    ode, tr, fp, y0, target = setup()
    _, grad, _ = loss_grad(tr, fp, y0, target)
    y0t = torch.tensor(y0, device="cuda")
    h = 1e-6
    for k in range(4):
        fpp, fpm = fp.copy(), fp.copy()
        fpp[:, k] *= 1 + h
        fpm[:, k] *= 1 - h
        lp = ((tr.run_forward(torch.tensor(fpp, device="cuda"), y0t) - target) ** 2).sum(0).cpu().numpy()
        lm = ((tr.run_forward(torch.tensor(fpm, device="cuda"), y0t) - target) ** 2).sum(0).cpu().numpy()
        fd = (lp - lm) / (2 * h * fp[:, k])
        np.testing.assert_allclose(grad[:, k], fd, rtol=2e-5, atol=1e-9 * np.abs(fd).max())


def test_checkpoint_spacing_does_not_change_gradient():
    ode, tr_a, fp, y0, target = setup(K=100)
    _, ga, _ = loss_grad(tr_a, fp, y0, target)
    _, tr_b, _, _, _ = setup(K=800)
    _, gb, _ = loss_grad(tr_b, fp, y0, target)
    assert np.array_equal(ga, gb)


def test_fp32_adjoint_close_to_fp64():
    ode, tr64, fp, y0, target = setup("double")
    _, g64, _ = loss_grad(tr64, fp, y0, target)
    _, tr32, _, _, _ = setup("single")
    _, g32, _ = loss_grad(tr32, fp, y0, target)
    rel = np.abs(g32 - g64).max() / np.abs(g64).max()
    assert rel < 1e-3, rel
