"""Adjoint of GRL1 traces (goss_b200.adjoint) against the FP64 tangent-linear reference.

The trace is the reference's user loop (forward(t0 + j*interval, interval),
V sampled after each interval); the loss a trace misfit.  Checks:

* the FP64 record kernel reproduces the oracle's trace (the reference's
  GRL1 semantics) to 1e-10;
* FP64 adjoint gradients w.r.t. the four conductance fields and the 19
  initial states equal the FP64 forward-mode tangent-linear reference
  (oracle/tangent) on every node;
* they equal central finite differences of the ORACLE's loss as far as
  finite differences resolve this model (1e-4 for the median over three
  steps: the sodium-gate rates switch branches discontinuously at V = -40 mV
  and the upstroke amplifies rounding);
* checkpoint spacing does not change the gradient;
* the FP32 adjoint against the FP64 tangent-linear reference.
"""
from __future__ import annotations

import numpy as np
import pytest

import goss_b200 as goss
import pyoracle
from goss_b200.adjoint import GRL1Trace, trace
from helpers import column_rel_err, oracle_state_traces, parity

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


def loss_grad(tr, fp, y0, target, with_states=False):
    import torch

    p = torch.tensor(fp, device="cuda", requires_grad=True)
    y = torch.tensor(y0, device="cuda", requires_grad=with_states)
    v = trace(tr, p, y)
    loss = ((v - target) ** 2).sum()
    loss.backward()
    if with_states:
        return float(loss.detach()), p.grad.cpu().numpy(), y.grad.cpu().numpy()
    return float(loss.detach()), p.grad.cpu().numpy(), v.detach().cpu().numpy()


def tangent_grad(ode, fp, y0, target, dirs):
    """Loss gradient along `dirs` from the FP64 tangent-linear reference."""
    tl = pyoracle.TangentTrace(ode.module.dir)
    tr, jac = tl.trace(y0, fp, ode._params, 0.0, INTERVAL, S, J, ode.state_names.index("V"), dirs)
    return np.einsum("jn,jnk->nk", 2 * (tr - target), jac)


def oracle_traces(ode, fp, y0):
    """Oracle (reference semantics) traces of V for every row of fp."""
    return oracle_state_traces(MODEL, F4, fp, y0, INTERVAL, S, J, ode.state_names.index("V"))


def test_record_trace_matches_oracle():
    import torch

    ode, tr, fp, y0, target = setup()
    v = tr.run_forward(torch.tensor(fp, device="cuda"), torch.tensor(y0, device="cuda")).cpu().numpy()
    ref = oracle_traces(ode, fp, y0)
    assert parity(v, ref, rtol=1e-10, atol=1e-12) <= 1.0


def test_fp64_adjoint_matches_tangent_linear():
    ode, tr, fp, y0, target = setup()
    _, gfp, gy0 = loss_grad(tr, fp, y0, target, with_states=True)
    n = ode.num_states
    ref = tangent_grad(ode, fp, y0, target.cpu().numpy(), list(range(n + 4)))
    assert column_rel_err(gfp, ref[:, n:]) < 1e-9
    assert column_rel_err(gy0, ref[:, :n]) < 1e-9


def test_adjoint_matches_oracle_central_differences():
    ode, tr, fp, y0, target = setup()
    _, grad, _ = loss_grad(tr, fp, y0, target)
    tgt = target.cpu().numpy()
    nodes = [0, 5, 11, 23]
    iv = ode.state_names.index("V")
    # a single step is either swamped by rounding amplified through the
    # upstroke (small h) or crosses a branch switch (large h) for some entry;
    # the median over three steps is robust to one bad estimate
    steps = (1e-4, 1e-5, 1e-6)
    fd = np.zeros((len(steps), len(nodes), 4))
    for i, h in enumerate(steps):
        for k in range(4):
            fpp, fpm = fp[nodes].copy(), fp[nodes].copy()
            fpp[:, k] *= 1 + h
            fpm[:, k] *= 1 - h
            lp = ((oracle_state_traces(MODEL, F4, fpp, y0[nodes], INTERVAL, S, J, iv) - tgt[:, nodes]) ** 2).sum(0)
            lm = ((oracle_state_traces(MODEL, F4, fpm, y0[nodes], INTERVAL, S, J, iv) - tgt[:, nodes]) ** 2).sum(0)
            fd[i, :, k] = (lp - lm) / (2 * h * fp[nodes, k])
    assert column_rel_err(grad[nodes], np.median(fd, axis=0)) < 1e-4


def test_checkpoint_spacing_does_not_change_gradient():
    ode, tr_a, fp, y0, target = setup(K=100)
    _, ga, _ = loss_grad(tr_a, fp, y0, target)
    _, tr_b, _, _, _ = setup(K=800)
    _, gb, _ = loss_grad(tr_b, fp, y0, target)
    # the recomputed segments are the recorded trajectory up to rounding
    assert np.abs(ga - gb).max() <= 1e-10 * np.abs(ga).max()


def test_fp32_adjoint_close_to_tangent_linear():
    ode, tr64, fp, y0, target = setup("double")
    ref = tangent_grad(ode, fp, y0, target.cpu().numpy(), [ode.num_states + k for k in range(4)])
    _, tr32, _, _, _ = setup("single")
    _, g32, _ = loss_grad(tr32, fp, y0, target)
    rel = column_rel_err(g32, ref)
    assert rel < 1e-3, rel


# ---------------------------------------------------------------------------
# both solvers, two models: record trace vs the oracle, FP64 adjoint vs the
# tangent-linear reference (fields and initial states), FP32 adjoint
# ---------------------------------------------------------------------------
CASES = [  # model, field parameters, solver, steps per 1 ms interval, intervals
    ("tentusscher_panfilov_2006_M_cell", F4, "GRL1", 100, 16),
    ("tentusscher_panfilov_2006_M_cell", F4, "RK4", 1000, 12),
    ("fitzhughnagumo", ["a", "b"], "RK4", 20, 40),
    ("fitzhughnagumo", ["a", "b"], "GRL1", 20, 40),
]
CASE_IDS = [f"{m.split('_')[0]}-{s}" for m, _, s, _, _ in CASES]


def case_setup(case, precision="double", nodes=16, K=None, seed=4, tape_segments=0):
    import torch
    from goss_b200.adjoint import SolverTrace

    model, fields, solver, steps, intervals = case
    ode = goss.ParameterizedODE(model, field_parameters=fields)
    rng = np.random.default_rng(seed)
    defaults = np.array([ode.get_parameter(p) for p in fields])
    fp = defaults[None, :] * np.exp(0.2 * rng.standard_normal((nodes, len(fields))))
    fp_target = defaults[None, :] * np.exp(0.2 * rng.standard_normal((nodes, len(fields))))
    y0 = ode.get_ic()[None, :] * (1 + rng.uniform(-0.02, 0.02, (nodes, ode.num_states)))
    K = K or steps * 4
    sld = (nodes + 255) // 256 * 256 + 256
    segment_bytes = K * ode.num_states * sld * (4 if precision == "single" else 8)
    tr = SolverTrace(ode, nodes, 1.0, steps, intervals, K, precision=precision, solver=solver,
                     tape_bytes=tape_segments * segment_bytes)
    target = tr.run_forward(torch.tensor(fp_target, device="cuda"), torch.tensor(y0, device="cuda")).clone()
    return ode, tr, fp, y0, target


def case_tangent(case, ode, fp, y0, target, dirs):
    model, fields, solver, steps, intervals = case
    tl = pyoracle.TangentTrace(ode.module.dir)
    iv = ode.state_names.index("V")
    trv, jac = tl.trace(y0, fp, ode._params, 0.0, 1.0, steps, intervals, iv, dirs, solver=solver)
    return trv, np.einsum("jn,jnk->nk", 2 * (trv - target), jac)


@pytest.mark.parametrize("case", CASES, ids=CASE_IDS)
def test_case_record_matches_oracle(case):
    import torch

    model, fields, solver, steps, intervals = case
    ode, tr, fp, y0, target = case_setup(case)
    v = tr.run_forward(torch.tensor(fp, device="cuda"), torch.tensor(y0, device="cuda")).cpu().numpy()
    ref = oracle_state_traces(model, fields, fp, y0, 1.0, steps, intervals, ode.state_names.index("V"),
                              solver=solver)
    assert parity(v, ref, rtol=1e-10, atol=1e-12) <= 1.0


@pytest.mark.parametrize("case", CASES, ids=CASE_IDS)
def test_case_fp64_adjoint_matches_tangent_linear(case):
    ode, tr, fp, y0, target = case_setup(case)
    _, gfp, gy0 = loss_grad(tr, fp, y0, target, with_states=True)
    n, nf = ode.num_states, len(case[1])
    _, ref = case_tangent(case, ode, fp, y0, target.cpu().numpy(), list(range(n + nf)))
    # the GPU and oracle trajectories agree to ~1e-10; the misfit residuals
    # (v - target) amplify that in relative terms, hence 1e-7, not 1e-10
    assert column_rel_err(gfp, ref[:, n:]) < 1e-7
    assert column_rel_err(gy0, ref[:, :n]) < 1e-7


@pytest.mark.parametrize("case", CASES, ids=CASE_IDS)
def test_case_fp32_adjoint_close_to_tangent_linear(case):
    ode, _, fp, y0, target = case_setup(case)
    nf = len(case[1])
    _, ref = case_tangent(case, ode, fp, y0, target.cpu().numpy(), [ode.num_states + k for k in range(nf)])
    _, tr32, _, _, _ = case_setup(case, "single")
    _, g32, _ = loss_grad(tr32, fp, y0, target)
    assert column_rel_err(g32, ref) < 2e-3


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("case", CASES, ids=CASE_IDS)
def test_case_tape_does_not_change_gradient(case, precision):
    """Segments taped by the record pass (all of them, or the last half) give
    the gradient of the recomputed segments: the tape holds the states the
    recompute reproduces."""
    ode, tr0, fp, y0, target = case_setup(case, precision)
    assert tr0.taped_segments == 0
    _, g0, s0 = loss_grad(tr0, fp, y0, target, with_states=True)
    num_cp = tr0.num_checkpoints
    for segments in (num_cp, num_cp // 2):
        _, tr, _, _, _ = case_setup(case, precision, tape_segments=segments)
        assert tr.taped_segments == segments
        _, g, s = loss_grad(tr, fp, y0, target, with_states=True)
        bar = 1e-10 if precision == "double" else 1e-6
        assert np.abs(g - g0).max() <= bar * np.abs(g0).max(), (segments, np.abs(g - g0).max() / np.abs(g0).max())
        assert np.abs(s - s0).max() <= bar * np.abs(s0).max(), (segments, np.abs(s - s0).max() / np.abs(s0).max())


def test_tape_size_arguments():
    from goss_b200.adjoint import SolverTrace

    ode = goss.ParameterizedODE(MODEL, field_parameters=F4)
    t = SolverTrace(ode, 24, INTERVAL, S, J, 400, tape_bytes=1 << 40)
    assert t.taped_segments == t.num_checkpoints == 4  # clamped to the segments there are
    assert SolverTrace(ode, 24, INTERVAL, S, J, 400, tape_bytes=1000).taped_segments == 0
    assert SolverTrace(ode, 24, INTERVAL, S, J, 400, tape_bytes="auto").taped_segments == 4
    with pytest.raises(TypeError):
        SolverTrace(ode, 24, INTERVAL, S, J, 400, tape_bytes=1.5)


def test_fp64_reverse_over_fp32_trajectory():
    """reverse_precision="double" over an FP32 record: the FP32 trajectory
    differentiated with FP64 step VJPs.  Its gradient sits between the FP32
    and the FP64 adjoints: against the FP64 adjoint it carries only the FP32
    trajectory's difference, against the FP32 adjoint only the FP32 reverse
    arithmetic's; each is bounded like the FP32 gradient's total error."""
    ode, tr64, fp, y0, target = setup("double")
    _, g64, _ = loss_grad(tr64, fp, y0, target)
    tr32 = GRL1Trace(ode, N, INTERVAL, S, J, 400, precision="single")
    _, g32, _ = loss_grad(tr32, fp, y0, target)
    trm = GRL1Trace(ode, N, INTERVAL, S, J, 400, precision="single", reverse_precision="double")
    _, gm, _ = loss_grad(trm, fp, y0, target)
    assert np.isfinite(gm).all()
    total = column_rel_err(g32, g64)
    assert column_rel_err(gm, g64) < 1e-3 and column_rel_err(g32, gm) < 1e-3, total
    with pytest.raises(ValueError):
        GRL1Trace(ode, N, INTERVAL, S, J, 400, precision="double", reverse_precision="single")
