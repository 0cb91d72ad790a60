"""Autotuner for the launch configuration of batches and single systems.

For a :class:`~goss_b200.batch.BatchSolver` it searches the tile size
(threads per block = nodes per tile), the persistent grid size, the tile
schedule (round-robin, an atomic work counter or prefetching CTAs) and the
order in which the populations' tiles are laid out (as given, or most
expensive first by the generator's operation census), timing each candidate
with CUDA events on the batch stream over a few graph-captured forwards (all
in one launch unless the candidate sets ``forwards_per_launch``).  For a single system it searches the
block size.  The states are saved before and restored after tuning, so
tuning does not advance the simulation.  Results are cached in
``goss_b200/_jit/autotune.json`` keyed by the device, the module and the
population sizes.
"""
from __future__ import annotations

import json
import threading
from pathlib import Path
from typing import Dict, List, Optional

import numpy as np

from .batch import BatchSolver
from .systemsolver import ODESystemSolver

CACHE = Path(__file__).resolve().parent / "_jit" / "autotune.json"
_lock = threading.Lock()

SMS = 148  # B200 streaming multiprocessors


def _device_name() -> str:
    try:
        import torch

        return torch.cuda.get_device_name(0)
    except Exception:
        return "cuda"


def _load_cache() -> Dict:
    try:
        return json.loads(CACHE.read_text())
    except Exception:
        return {}


def _store(key: str, value: Dict) -> None:
    with _lock:
        cache = _load_cache()
        cache[key] = value
        CACHE.parent.mkdir(parents=True, exist_ok=True)
        CACHE.write_text(json.dumps(cache, indent=1, sort_keys=True))


def _cost(system: ODESystemSolver) -> float:
    """Relative cost of one forward of a population (op census x nodes x steps)."""
    md = system.ode.module.meta
    census = md["op_census"]["linearized" if type(system.solver).__name__.startswith("GRL") else "rhs"]
    per_eval = sum(census.values()) + 7 * (census["exp"] + census["div"])
    evals = {"RK4": 4, "GRL2": 2}.get(type(system.solver).__name__, 1)
    return float(per_eval * evals * system.num_nodes)


def tune_batch(batch: BatchSolver, interval: float, t0: float = 0.0, steps: int = 3, use_graph: bool = True,
               use_cache: bool = True, candidates: Optional[List[Dict]] = None) -> Dict:
    """Pick and apply the fastest configuration; returns it with its time."""
    key = json.dumps(dict(device=_device_name(), module=batch.module.meta["name"],
                          pops=[(s.ode.module.meta["variant"], type(s.solver).__name__, s.num_nodes)
                                for s in batch.systems],
                          interval=interval, precision=batch.systems[0].precision), sort_keys=True)
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            batch.set_config(hit["block"], hit["grid"], hit["schedule"], hit["order"],
                             hit.get("forwards_per_launch", 0))
            return dict(hit, cached=True)
    saved = [s.states for s in batch.systems]
    costs = [_cost(s) for s in batch.systems]
    by_cost = list(np.argsort(costs)[::-1])
    if candidates is None:
        candidates = []
        for block in (64, 128):
            for schedule in (0, 1):
                for grid_mult in (0, 2, 4, 8):
                    for order in (None, [int(i) for i in by_cost]):
                        grid = 0 if grid_mult == 0 else SMS * grid_mult * (128 // block)
                        if schedule == 1 and grid == 0:
                            continue  # a work counter only helps a persistent grid
                        candidates.append(dict(block=block, grid=grid, schedule=schedule, order=order))
            for order in (None, [int(i) for i in by_cost]):   # persistent, prefetching
                candidates.append(dict(block=block, grid=0, schedule=2, order=order))
    best = None
    try:
        for c in candidates:
            batch.set_config(**c)
            batch.time(t0, interval, 1, use_graph=False)  # warm-up
            ms = batch.time(t0, interval, steps, use_graph=use_graph)
            if best is None or ms < best["ms"]:
                best = dict(c, ms=ms)
    finally:
        for s, y in zip(batch.systems, saved):
            s.set_states(y)
    batch.set_config(best["block"], best["grid"], best["schedule"], best["order"], best.get("forwards_per_launch", 0))
    _store(key, best)
    return dict(best, cached=False, tried=len(candidates))


def tune_system(system: ODESystemSolver, interval: float, t0: float = 0.0, steps: int = 3,
                use_cache: bool = True) -> Dict:
    """Block size of a single system's solver kernel."""
    import time

    key = json.dumps(dict(device=_device_name(), variant=system.ode.module.meta["variant"],
                          solver=type(system.solver).__name__, nodes=system.num_nodes, interval=interval,
                          precision=system.precision), sort_keys=True)
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            system.set_block_size(hit["block"])
            return dict(hit, cached=True)
    saved = system.states
    best = None
    try:
        # the implicit kernels run in block lockstep, in blocks of up to 256
        lockstep = type(system.solver).__name__ in ("ThetaSolver", "ImplicitEuler", "ESDIRK23a")
        for block in (32, 64, 96, 128) + ((192, 256) if lockstep else ()):
            system.set_block_size(block)
            system.forward(t0, interval)
            system.synchronize()
            w0 = time.perf_counter()
            for k in range(steps):
                system.forward_async(t0 + k * interval, interval)
            system.synchronize()
            ms = (time.perf_counter() - w0) * 1e3
            if best is None or ms < best["ms"]:
                best = dict(block=block, ms=ms)
    finally:
        system.set_states(saved)
    system.set_block_size(best["block"])
    _store(key, best)
    return dict(best, cached=False)
