"""Heterogeneous populations in one persistent kernel launch.

``BatchSolver([system_a, system_b, ...])`` advances several
:class:`~goss_b200.systemsolver.ODESystemSolver` populations -- different
models, explicit solvers and sizes -- with ONE kernel launch per forward,
optionally replaying a captured CUDA graph of many forwards.  The
populations keep their own states, field parameters and parameters; the
batch only schedules them.  The reference has no such object: it runs one
``ODESystemSolver`` per population (one per subdomain in
``python/goss/dolfinutils.py:519-530``).

The batch module (the kernel for the set of (model variant, solver) kinds)
is taken from the shipped modules in ``goss_b200/batches/`` or generated and
compiled into ``goss_b200/_jit/`` on first use.
"""
from __future__ import annotations

import ctypes as C
import json
import threading
from pathlib import Path
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _capi
from .build import build_batch
from .codegen.batchgen import batch_name, write_batch
from .systemsolver import ODESystemSolver

PKG = Path(__file__).resolve().parent
BATCH_DIR = PKG / "batches"
JIT_DIR = PKG / "_jit"

_lock = threading.Lock()
_loaded: Dict[str, "BatchModule"] = {}


BatchDesc = _capi.BatchDesc


def _lib():
    return _capi.lib()


def _check(rc, handle=None):
    if rc == _capi.GOSS_OK:
        return
    msg = _lib().goss_batch_last_error(handle).decode() if handle else ""
    if not msg:
        msg = _capi.lib().goss_last_error().decode()
    if rc == _capi.GOSS_ERR_ARGUMENT:
        raise ValueError(msg)
    raise _capi.GossError(rc, msg)


class BatchModule:
    def __init__(self, bdir: Path):
        self.dir = Path(bdir)
        self.meta = json.loads((self.dir / "batch.json").read_text())
        so = build_batch(self.dir)
        self._lib = C.CDLL(str(so))
        f = getattr(self._lib, f"goss_b200_batch_{self.meta['name']}")
        f.restype = C.POINTER(BatchDesc)
        self.desc = f()
        if self.desc.contents.abi_version != _capi.ABI_VERSION:
            raise _capi.ExtensionMissingError(f"{so}: batch descriptor has the wrong ABI version")

    @property
    def kinds(self) -> List[Tuple[str, str]]:
        return [tuple(k) for k in self.meta["kinds"]]


def _kind_key(system: ODESystemSolver) -> Tuple[str, str]:
    vdir = Path(system.ode.module.dir).resolve().relative_to(PKG).as_posix()
    return (vdir, type(system.solver).__name__)


def find_module(kinds: Sequence[Tuple[str, str]]) -> Tuple["BatchModule", List[int]]:
    """A batch module whose kinds include every requested kind."""
    want = [tuple(k) for k in kinds]
    candidates = sorted(BATCH_DIR.glob("*/batch.json")) + sorted(JIT_DIR.glob("batch_*/batch.json"))
    for bj in candidates:
        meta = json.loads(bj.read_text())
        have = [tuple(k) for k in meta["kinds"]]
        if all(k in have for k in want):
            return load_module(bj.parent), [have.index(k) for k in want]
    name = batch_name(want)
    bdir = JIT_DIR / name
    with _lock:
        write_batch(name, [(PKG / v, s) for v, s in want], bdir, PKG)
    return load_module(bdir), list(range(len(want)))


def load_module(bdir: Path) -> BatchModule:
    key = str(Path(bdir).resolve())
    with _lock:
        mod = _loaded.get(key)
        if mod is None:
            mod = BatchModule(Path(bdir))
            _loaded[key] = mod
        return mod


class BatchSolver:
    """Several node populations advanced by one kernel per forward."""

    def __init__(self, systems: Sequence[ODESystemSolver], precision: Optional[str] = None):
        systems = list(systems)
        if not systems:
            raise ValueError("a batch needs at least one population")
        from .solvers import ImplicitODESolver

        for s in systems:
            if isinstance(s.solver, ImplicitODESolver):
                raise ValueError("batches run explicit solvers (ExplicitEuler, RK4, GRL1, GRL2)")
        prec = precision or systems[0].precision
        if any(s.precision != prec for s in systems):
            raise ValueError("all populations of a batch share one precision")
        self.systems = systems
        keys = [_kind_key(s) for s in systems]
        uniq = list(dict.fromkeys(keys))
        self.module, idx = find_module(uniq)
        kinds = np.array([idx[uniq.index(k)] for k in keys], dtype=np.int32)
        handles = (C.c_void_p * len(systems))(*[s._h.value for s in systems])
        for s in systems:
            s._sync_params()
        h = C.c_void_p()
        _check(_lib().goss_batch_create(self.module.desc, handles, kinds.ctypes.data_as(C.POINTER(C.c_int32)),
                                        len(systems), _capi.GOSS_FP32 if prec == "single" else _capi.GOSS_FP64,
                                        C.byref(h)))
        self._h = h
        self._kinds = kinds
        self.config = dict(block=128, grid=0, schedule=1, order=None, forwards_per_launch=0)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib().goss_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_config(self, block: int = 128, grid: int = 0, schedule: int = 1, order: Optional[Sequence[int]] = None,
                   forwards_per_launch: int = 0):
        """Launch configuration: nodes per tile, persistent grid (0: a block
        per tile), tile schedule, population order, and how many consecutive
        forwards of a captured graph one launch performs (0: all of them, the
        states kept on chip in between; 1: a launch per forward)."""
        o = None if order is None else (C.c_uint32 * len(order))(*order)
        _check(_lib().goss_batch_set_config(self._h, int(block), int(grid), int(schedule), o), self._h)
        _check(_lib().goss_batch_set_forwards_per_launch(self._h, int(forwards_per_launch)), self._h)
        self.config = dict(block=int(block), grid=int(grid), schedule=int(schedule),
                           order=None if order is None else list(order), forwards_per_launch=int(forwards_per_launch))

    def _sync(self):
        for s in self.systems:
            s._sync_params()

    def forward(self, t: float, interval: float) -> None:
        self._sync()
        _check(_lib().goss_batch_forward(self._h, float(t), float(interval)), self._h)

    def capture(self, t0: float, interval: float, num_steps: int) -> None:
        """Record num_steps forwards (t0 + k*interval) into a CUDA graph,
        ``config["forwards_per_launch"]`` of them per launch."""
        self._sync()
        _check(_lib().goss_batch_capture(self._h, float(t0), float(interval), int(num_steps)), self._h)

    def replay(self) -> None:
        _check(_lib().goss_batch_replay(self._h), self._h)

    def time(self, t0: float, interval: float, num_steps: int, use_graph: bool = True) -> float:
        """Device time in ms of num_steps forwards (CUDA events); states advance."""
        self._sync()
        ms = C.c_float(0.0)
        _check(_lib().goss_batch_time(self._h, float(t0), float(interval), int(num_steps), int(bool(use_graph)),
                                      C.byref(ms)), self._h)
        return float(ms.value)

    @property
    def total_nodes(self) -> int:
        return sum(s.num_nodes for s in self.systems)
