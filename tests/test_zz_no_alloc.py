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


def _host_eval(ode, what, states, times, field_params=None):
    return ode._eval(what, states, times, _capi.GOSS_FP64, field_params)


def _noalloc_eval(ode, what, states, times, field_params=None, precision=_capi.GOSS_FP64):
    import torch

    n = ode.num_states
    width = {0: n, 1: 2 * n, 2: len(ode.monitored_names)}[what]
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
