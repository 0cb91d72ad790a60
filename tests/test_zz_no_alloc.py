"""The allocation-free evaluation entry point, ``goss_model_eval_noalloc``.

It serves callers that must not have this library call ``cudaMalloc``: a
process whose GPU memory belongs to another allocator (a framework's caching
allocator that reserved the device, or a fixed memory budget), where a
library allocation would fail, stall on that allocator or fragment its pool.
Such a caller passes device buffers for the inputs and outputs; the library
keeps its working arrays in a fixed device array.

The test calls it through the C ABI twice in a row with different inputs and
checks each result against the allocating ``goss_model_eval``.  The device
buffers are made by torch here only because a test needs some device memory
to hand over.  This file is named to be collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import goss_b200 as goss
from goss_b200 import _capi
from helpers import parity

pytestmark = pytest.mark.gpu


def _host_eval(ode, what, states, times, field_params=None, precision=_capi.GOSS_FP64):
    return ode._eval(what, states, times, precision, field_params)


def _noalloc_eval(ode, what, states, times, field_params=None, precision=_capi.GOSS_FP64):
    import torch

    n = ode.num_states
    width = {0: n, 1: 2 * n, 2: len(ode.monitored_names), 3: n * n}[what]
    d_states = torch.as_tensor(np.ascontiguousarray(states), device="cuda")
    d_times = torch.as_tensor(np.ascontiguousarray(times), device="cuda")
    d_fp = None if field_params is None else torch.as_tensor(np.ascontiguousarray(field_params), device="cuda")
    d_out = torch.full((states.shape[0], width), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    rc = _capi.lib().goss_model_eval_noalloc(
        ode.module.desc, what, precision, _capi.ptr(ode._params), d_states.data_ptr(),
        d_fp.data_ptr() if d_fp is not None else None, d_times.data_ptr(), states.shape[0], d_out.data_ptr(),
        C.c_void_p(stream.cuda_stream))
    _capi.check(rc)
    return d_out.cpu().numpy()


def test_noalloc_matches_allocating_eval_two_calls():
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell", field_parameters=["g_Kr", "g_Ks", "g_CaL",
                                                                                       "g_to"])
    rng = np.random.default_rng(17)
    for call in range(2):  # the scratch keeps the previous call's contents
        count = 1000 + 333 * call
        states = ode.get_ic()[None, :] * (1 + rng.uniform(-0.2, 0.2, (count, ode.num_states)))
        times = rng.uniform(0, 20, count)
        fp = np.array([0.153, 0.098, 3.98e-05, 0.294])[None, :] * np.exp(0.2 * rng.standard_normal((count, 4)))
        for what in (0, 1):
            ref = _host_eval(ode, what, states, times, fp)
            got = _noalloc_eval(ode, what, states, times, fp)
            assert np.isfinite(got).all()
            assert parity(got, ref, rtol=1e-10, atol=1e-12) <= 1.0


def test_noalloc_default_field_parameters_and_monitored():
    ode = goss.ParameterizedODE("fitzhughnagumo", monitored=["p_42", "p_V"])
    rng = np.random.default_rng(3)
    for call in range(2):
        states = ode.get_ic()[None, :] * (1 + rng.uniform(-0.1, 0.1, (257, 2)))
        times = rng.uniform(0, 5, 257)
        for what in (0, 1, 2):
            ref = _host_eval(ode, what, states, times)
            got = _noalloc_eval(ode, what, states, times)
            assert parity(got, ref, rtol=1e-10, atol=1e-12) <= 1.0


def test_noalloc_rejects_oversize_requests():
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell")
    cap = _capi.lib().goss_model_eval_noalloc_capacity()
    count = int(cap // (3 * ode.num_states)) + 64  # does not fit for what=1
    states = np.tile(ode.get_ic(), (count, 1))
    times = np.zeros(count)
    with pytest.raises(ValueError, match="fixed scratch holds"):
        _noalloc_eval(ode, 1, states, times)


def test_noalloc_fp32_and_analytic_jacobian():
    """FP32 arithmetic (the float instantiation of the evaluation kernel) and
    what = 3, the analytic Jacobian (n*n values per state) of a model
    generated with it, each against the allocating call in the same precision."""
    rng = np.random.default_rng(29)
    ode = goss.ParameterizedODE("tentusscher_panfilov_2006_M_cell", field_parameters=["g_Kr", "g_Ks", "g_CaL",
                                                                                       "g_to"])
    for call in range(2):
        count = 640 + 97 * call
        states = ode.get_ic()[None, :] * (1 + rng.uniform(-0.2, 0.2, (count, ode.num_states)))
        times = rng.uniform(0, 20, count)
        fp = np.array([0.153, 0.098, 3.98e-05, 0.294])[None, :] * np.exp(0.2 * rng.standard_normal((count, 4)))
        for what in (0, 1):
            ref = _host_eval(ode, what, states, times, fp, _capi.GOSS_FP32)
            got = _noalloc_eval(ode, what, states, times, fp, _capi.GOSS_FP32)
            assert np.isfinite(got).all()
            assert parity(got, ref, rtol=1e-10, atol=1e-12) <= 1.0
    jac = goss.ParameterizedODE("tentusscher_2004_mcell", field_parameters=["g_Kr", "g_CaL"],
                                code_params={"generate_jacobian": True})
    assert jac.has_jacobian
    for call in range(2):
        count = 300 + 41 * call
        states = jac.get_ic()[None, :] * (1 + rng.uniform(-0.1, 0.1, (count, jac.num_states)))
        times = rng.uniform(0, 5, count)
        fp = np.array([jac.get_parameter("g_Kr"), jac.get_parameter("g_CaL")])[None, :] * \
            (1 + rng.uniform(-0.05, 0.05, (count, 2)))
        ref = _host_eval(jac, 3, states, times, fp)
        got = _noalloc_eval(jac, 3, states, times, fp)
        assert got.shape == (count, jac.num_states ** 2)
        assert parity(got, ref, rtol=1e-10, atol=1e-12) <= 1.0


def test_noalloc_field_parameters_from_the_parameter_values():
    """A model with field parameters called without field_params: every node
    takes the current (here non-default) parameter values, as the allocating
    call does."""
    ode = goss.ParameterizedODE("fitzhughnagumo", field_parameters=["a", "b"])
    ode.set_parameter("a", 0.17)
    ode.set_parameter("b", 0.009)
    rng = np.random.default_rng(31)
    for call in range(2):
        count = 129 + call
        states = ode.get_ic()[None, :] * (1 + rng.uniform(-0.1, 0.1, (count, 2)))
        times = rng.uniform(0, 5, count)
        explicit = np.tile([0.17, 0.009], (count, 1))
        for what in (0, 1):
            ref = _host_eval(ode, what, states, times, explicit)
            assert np.array_equal(_host_eval(ode, what, states, times), ref)
            got = _noalloc_eval(ode, what, states, times)
            assert parity(got, ref, rtol=1e-10, atol=1e-12) <= 1.0
