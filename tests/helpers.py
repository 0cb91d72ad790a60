"""Test helpers: model variants and the oracle (CPU checker)."""
from __future__ import annotations

import json
from functools import lru_cache
from pathlib import Path

import numpy as np

import pyoracle
from goss_b200 import models

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"


def variant_dir(name: str, field_parameters=(), jacobian: bool = False) -> Path:
    d = models.find_variant(name, list(field_parameters), jacobian=jacobian)
    assert d is not None, f"no shipped variant {name} {field_parameters}" + (" with the Jacobian" if jacobian else "")
    return d


def meta(vdir: Path) -> dict:
    return json.loads((vdir / "model.json").read_text())


@lru_cache(maxsize=None)
def oracle_model(name: str, field_parameters=(), jacobian: bool = False) -> pyoracle.OracleModel:
    vdir = variant_dir(name, field_parameters, jacobian)
    md = meta(vdir)
    return pyoracle.OracleModel(pyoracle.build_oracle(vdir, md["ident"]), md["ident"])


def ref_system(name: str, solver: str, num_nodes: int, field_parameters=(), jacobian: bool = False, **sp):
    """The reference's compiled solvers, or None when oracle/_ref is not built."""
    vdir = variant_dir(name, field_parameters, jacobian)
    if not pyoracle.ref_available():
        return None
    plug = pyoracle.build_ref_plugin(vdir)
    if plug is None or not plug.exists():
        return None
    om = oracle_model(name, tuple(field_parameters), jacobian)
    return pyoracle.RefSystem(plug, meta(vdir)["class_name"], solver, num_nodes, om.solver_params(solver, **sp))


def perturbed_states(ic, num_nodes, rng, spread=0.05):
    ic = np.asarray(ic, dtype=np.float64)
    return ic[None, :] * (1.0 + rng.uniform(-spread, spread, (num_nodes, ic.size)))


def rel_err(a, b, floor=1e-12):
    """max |a-b| / max(|b|, floor): relative error with an absolute floor."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.maximum(np.abs(b), floor)
    return float(np.max(np.abs(a - b) / den)) if a.size else 0.0


def parity(a, b, rtol=1e-10, atol=1e-12):
    """Worst ratio |a-b| / (atol + rtol*|b|); parity holds when it is <= 1.

    rtol is the relative bar for FP64 states; atol = 1e-12 is the absolute
    floor for states that decay towards zero (e.g. the h and j gates at
    ~1e-10 after the upstroke), whose relative error says nothing."""
    a = np.asarray(a)
    b = np.asarray(b)
    if not a.size:
        return 0.0
    if not (np.isfinite(a) == np.isfinite(b)).all():
        return float("inf")
    m = np.isfinite(b)
    return float(np.max(np.abs(a[m] - b[m]) / (atol + rtol * np.abs(b[m])))) if m.any() else 0.0


def parity_scaled(a, b, rtol=1e-10, atol=1e-12, floor=0.01):
    """parity() with each state's magnitude floored at `floor` times that
    state's largest magnitude over the compared rows: |a-b| / (atol + rtol *
    max(|b|, floor * max|b[:, i]|)).  For states that pass through zero (the
    membrane potential during an upstroke), where a relative error compares
    rounding with a value that happens to be near 0."""
    a = np.atleast_2d(np.asarray(a))
    b = np.atleast_2d(np.asarray(b))
    if not a.size:
        return 0.0
    if not (np.isfinite(a) == np.isfinite(b)).all():
        return float("inf")
    scale = floor * np.nanmax(np.abs(np.where(np.isfinite(b), b, np.nan)), axis=0, keepdims=True)
    den = atol + rtol * np.maximum(np.abs(b), scale)
    m = np.isfinite(b)
    return float(np.max(np.abs(a[m] - b[m]) / den[m])) if m.any() else 0.0


def oracle_state_traces(name, field_parameters, fp, y0, interval, steps_per_interval, num_intervals, state_index,
                        t0=0.0, solver="GRL1"):
    """Oracle (reference semantics) traces [J, nodes] of one state: the loop
    forward(t0 + j*interval, interval) of an explicit solver, sampled after
    every interval."""
    om = oracle_model(name, tuple(field_parameters))
    y0 = np.atleast_2d(np.asarray(y0, dtype=np.float64))
    o = pyoracle.OracleSystem(om, solver, y0.shape[0], ldt=interval / steps_per_interval)
    o.states[:] = y0
    if om.nfp:
        o.field_params[:] = fp
    out = np.zeros((num_intervals, y0.shape[0]))
    for j in range(num_intervals):
        o.forward(t0 + j * interval, interval)
        out[j] = o.states[:, state_index]
    return out


def column_rel_err(a, b):
    """max over rows of |a-b| / max |b| per column, worst column: the error of
    a gradient [nodes, inputs] relative to each input's gradient scale."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b).max(axis=0) / np.maximum(np.abs(b).max(axis=0), 1e-300)))
