"""Test infrastructure -- NOT part of the product path.

ctypes access to the oracle: the C restatement (``goss_oracle.c`` plus a
generated model C file, built into ``oracle/_build/<variant>/liboracle.so``)
and, when it has been built, the reference's own solvers
(``oracle/_ref/``, see ``oracle/Makefile`` and ``oracle/ref_driver.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
REFDIR = HERE / "_ref"

SOLVERS = {"ExplicitEuler": 0, "RK4": 1, "GRL1": 2, "GRL2": 3, "ThetaSolver": 4, "ESDIRK23a": 5,
           "RL1": 6, "RL2": 7, "RK2": 8, "ImplicitEuler": 9}

_dp = C.POINTER(C.c_double)


class _Model(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("num_states", C.c_int),
        ("num_params", C.c_int),
        ("num_field_params", C.c_int),
        ("field_param_index", C.POINTER(C.c_uint)),
        ("rhs", C.CFUNCTYPE(None, _dp, C.c_double, _dp, _dp)),
        ("linearized", C.CFUNCTYPE(None, _dp, C.c_double, _dp, _dp, _dp, C.c_int)),
        ("ic", _dp),
        ("default_params", _dp),
        ("linear_terms", C.POINTER(C.c_ubyte)),
        ("jacobian", C.CFUNCTYPE(None, _dp, C.c_double, _dp, _dp)),
    ]


class SolverParams(C.Structure):
    _fields_ = [
        ("ldt", C.c_double),
        ("delta", C.c_double),
        ("eta_0", C.c_double),
        ("kappa", C.c_double),
        ("relative_tolerance", C.c_double),
        ("max_relative_previous_residual", C.c_double),
        ("max_iterations", C.c_int),
        ("always_recompute_jacobian", C.c_int),
        ("num_refinements_without_always_recomputing_jacobian", C.c_int),
        ("min_dt", C.c_double),
        ("theta", C.c_double),
    ]


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def build_oracle(variant_dir: Path, ident: str, force: bool = False) -> Path:
    """Compile goss_oracle.c + the variant's generated C model into a .so."""
    out = BUILD / variant_dir.name / "liboracle.so"
    src = variant_dir / "oracle_model.c"
    deps = [src, HERE / "goss_oracle.c", HERE / "goss_oracle.h"]
    if not force and out.exists() and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return out
    out.parent.mkdir(parents=True, exist_ok=True)
    cmd = [_cc("gcc"), "-O2", "-fPIC", "-shared", "-fopenmp", "-std=c11", f"-I{HERE}", str(HERE / "goss_oracle.c"),
           str(src), "-lm", "-o", str(out)]
    subprocess.run(cmd, check=True)
    return out


class OracleModel:
    """Single-state evaluation of a generated model through the C restatement."""

    def __init__(self, lib_path: Path, ident: str):
        self.lib = C.CDLL(str(lib_path))
        getter = getattr(self.lib, f"oracle_model_{ident}")
        getter.restype = C.POINTER(_Model)
        self.ptr = getter()
        self.m = self.ptr.contents
        self.n = self.m.num_states
        self.np = self.m.num_params
        self.nfp = self.m.num_field_params
        self.lib.oracle_system_create.restype = C.c_void_p
        self.lib.oracle_system_create.argtypes = [C.POINTER(_Model), C.c_int, C.POINTER(SolverParams), C.c_uint32]
        self.lib.oracle_system_destroy.argtypes = [C.c_void_p]
        for f in ("oracle_system_states", "oracle_system_field_params", "oracle_system_params"):
            getattr(self.lib, f).restype = _dp
            getattr(self.lib, f).argtypes = [C.c_void_p]
        self.lib.oracle_system_forward.restype = C.c_int
        self.lib.oracle_system_forward.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        self.lib.oracle_system_counters.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 3
        self.lib.oracle_default_solver_params.argtypes = [C.c_int, C.POINTER(SolverParams)]
        self.lib.oracle_compute_jacobian.argtypes = [C.POINTER(_Model), _dp, _dp, C.c_double, _dp, _dp, _dp]
        self.lib.oracle_lu_factorize.argtypes = [C.c_int, _dp]
        self.lib.oracle_forward_backward_subst.argtypes = [C.c_int, _dp, _dp, _dp]

    @property
    def ic(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.m.ic, shape=(self.n,)).copy()

    @property
    def default_params(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.m.default_params, shape=(max(self.np, 1),))[: self.np].copy()

    def rhs(self, y, t, params=None) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        p = self.default_params if params is None else np.ascontiguousarray(params, dtype=np.float64)
        out = np.zeros(self.n)
        self.m.rhs(_ptr(y), float(t), _ptr(p), _ptr(out))
        return out

    def linearized(self, y, t, params=None, only_linear=False):
        y = np.ascontiguousarray(y, dtype=np.float64)
        p = self.default_params if params is None else np.ascontiguousarray(params, dtype=np.float64)
        lin = np.zeros(self.n)
        rhs = np.zeros(self.n)
        self.m.linearized(_ptr(y), float(t), _ptr(p), _ptr(lin), _ptr(rhs), int(only_linear))
        return lin, rhs

    def jacobian(self, y, t, params=None) -> np.ndarray:
        y = np.array(y, dtype=np.float64)
        p = self.default_params if params is None else np.ascontiguousarray(params, dtype=np.float64)
        jac = np.zeros((self.n, self.n))
        f1, f2 = np.zeros(self.n), np.zeros(self.n)
        self.lib.oracle_compute_jacobian(self.ptr, _ptr(p), _ptr(y), float(t), _ptr(jac), _ptr(f1), _ptr(f2))
        return jac

    def lu_factorize(self, mat: np.ndarray) -> None:
        """ODE::lu_factorize restated (dense, in place)."""
        assert mat.dtype == np.float64 and mat.flags.c_contiguous and mat.shape == (self.n, self.n)
        self.lib.oracle_lu_factorize(self.n, _ptr(mat))

    def forward_backward_subst(self, mat: np.ndarray, b: np.ndarray) -> np.ndarray:
        x = np.zeros(self.n)
        self.lib.oracle_forward_backward_subst(self.n, _ptr(np.ascontiguousarray(mat)),
                                               _ptr(np.ascontiguousarray(b, dtype=np.float64)), _ptr(x))
        return x

    def solver_params(self, solver: str, **overrides) -> SolverParams:
        sp = SolverParams()
        self.lib.oracle_default_solver_params(SOLVERS[solver], C.byref(sp))
        for k, v in overrides.items():
            setattr(sp, k, v)
        return sp


class OracleSystem:
    """Multi-node FP64 CPU solve (restatement of ODESystemSolver::forward)."""

    def __init__(self, model: OracleModel, solver: str, num_nodes: int, **solver_params):
        self.model = model
        self.solver = solver
        self.N = int(num_nodes)
        self.sp = model.solver_params(solver, **solver_params)
        self.h = model.lib.oracle_system_create(model.ptr, SOLVERS[solver], C.byref(self.sp), self.N)
        n, nfp = model.n, model.nfp
        self.states = np.ctypeslib.as_array(model.lib.oracle_system_states(self.h), shape=(self.N, n))
        self.field_params = np.ctypeslib.as_array(model.lib.oracle_system_field_params(self.h),
                                                  shape=(self.N, max(nfp, 1)))[:, :nfp]
        self.params = np.ctypeslib.as_array(model.lib.oracle_system_params(self.h), shape=(max(model.np, 1),))

    def forward(self, t: float, interval: float, threads: Optional[int] = None) -> int:
        if threads is None:
            threads = os.cpu_count() or 1
        return self.model.lib.oracle_system_forward(self.h, float(t), float(interval), int(threads))

    def counters(self):
        jc = np.zeros(self.N, dtype=np.int64)
        rj = np.zeros(self.N, dtype=np.int64)
        ac = np.zeros(self.N, dtype=np.int64)
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))
        self.model.lib.oracle_system_counters(self.h, p(jc), p(rj), p(ac))
        return jc, rj, ac

    def __del__(self):
        try:
            self.model.lib.oracle_system_destroy(self.h)
        except Exception:
            pass


# ---------------------------------------------------------------------------
# the reference's own solvers (oracle/_ref, built by oracle/Makefile)
# ---------------------------------------------------------------------------
TANGENT = HERE / "tangent"


def build_tangent(variant_dir: Path, force: bool = False) -> Path:
    """Compile tangent/tangent_trace.cpp over a variant's generated device.cuh."""
    import json

    variant_dir = Path(variant_dir).resolve()
    struct = "M_" + json.loads((variant_dir / "model.json").read_text())["variant"]
    out = BUILD / "tangent" / variant_dir.name / "libtangent.so"
    deps = [variant_dir / "device.cuh", TANGENT / "tangent_trace.cpp", TANGENT / "goss_device_math.cuh"]
    if not force and out.exists() and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return out
    out.parent.mkdir(parents=True, exist_ok=True)
    tmp = out.with_suffix(f".so.{os.getpid()}.tmp")
    subprocess.run([_cc("g++"), "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", f"-I{TANGENT}",
                    f"-I{variant_dir}", f"-DGOSS_TANGENT_MODEL={struct}", str(TANGENT / "tangent_trace.cpp"),
                    "-o", str(tmp)], check=True)
    os.replace(tmp, out)
    return out


class TangentTrace:
    """FP64 forward-mode tangent-linear GRL1 / RK4 traces of one model variant.

    ``trace(states0 [N, n], field_params [N, nfp], params, t0, interval,
    steps_per_interval, num_intervals, trace_state, dirs, solver="GRL1")``
    returns the trace [J, N] and its Jacobian [J, N, len(dirs)] with respect
    to the inputs ``dirs`` (index < n: an initial state; else field parameter
    index - n).
    """

    def __init__(self, variant_dir: Path):
        self.lib = C.CDLL(str(build_tangent(variant_dir)))
        self.lib.tangent_trace.restype = C.c_int
        self.lib.tangent_trace.argtypes = [
            C.c_int, C.c_uint32, _dp, _dp, _dp, C.c_double, C.c_double, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
            C.POINTER(C.c_uint32), C.c_double, _dp, _dp]
        self.n = self.lib.tangent_num_states()
        self.nfp = self.lib.tangent_num_field_params()
        self.num_params = self.lib.tangent_num_params()
        self.num_derived = self.lib.tangent_num_derived()

    def _pvec(self, params):
        P = np.zeros(self.num_params + self.num_derived)
        P[: self.num_params] = params
        return P

    def jvp(self, y, F, params, time, ydot, Fdot):
        """(linear, rhs, linear_dot, rhs_dot) of one evaluation along (ydot, Fdot)."""
        f64 = lambda a, n: np.ascontiguousarray(np.resize(np.asarray(a, dtype=np.float64), max(n, 1)))
        y, ydot = f64(y, self.n), f64(ydot, self.n)
        F, Fdot = f64(F if self.nfp else [0.0], self.nfp), f64(Fdot if self.nfp else [0.0], self.nfp)
        out = [np.zeros(self.n) for _ in range(4)]
        self.lib.tangent_jvp(_ptr(y), _ptr(F), _ptr(self._pvec(params)), C.c_double(time), _ptr(ydot), _ptr(Fdot),
                             *[_ptr(o) for o in out])
        return tuple(out)

    def vjp(self, y, F, params, time, abar, bbar):
        """(ybar, Fbar) of one evaluation from the generated reverse sweep."""
        f64 = lambda a, n: np.ascontiguousarray(np.resize(np.asarray(a, dtype=np.float64), max(n, 1)))
        y, abar, bbar = f64(y, self.n), f64(abar, self.n), f64(bbar, self.n)
        F = f64(F if self.nfp else [0.0], self.nfp)
        ybar, Fbar = np.zeros(self.n), np.zeros(max(self.nfp, 1))
        self.lib.tangent_vjp(_ptr(y), _ptr(F), _ptr(self._pvec(params)), C.c_double(time), _ptr(abar), _ptr(bbar),
                             _ptr(ybar), _ptr(Fbar))
        return ybar, Fbar[: self.nfp]

    def trace(self, states0, field_params, params, t0, interval, steps_per_interval, num_intervals, trace_state,
              dirs, solver="GRL1", delta=1e-8):
        y0 = np.ascontiguousarray(states0, dtype=np.float64).reshape(-1, self.n)
        N = y0.shape[0]
        fp = np.ascontiguousarray(field_params if self.nfp else np.zeros((N, 1)), dtype=np.float64)
        P = self._pvec(params)
        d = np.ascontiguousarray(dirs, dtype=np.uint32)
        tr = np.zeros((num_intervals, N))
        jac = np.zeros((num_intervals, N, len(d)))
        rc = self.lib.tangent_trace({"GRL1": 0, "RK4": 1}[solver], N, _ptr(y0), _ptr(fp), _ptr(P), t0, interval, steps_per_interval,
                                         num_intervals, trace_state, len(d),
                                         d.ctypes.data_as(C.POINTER(C.c_uint32)), delta, _ptr(tr), _ptr(jac))
        if rc != 0:
            raise ValueError("tangent_trace: bad arguments")
        return tr, jac


def reference_dir() -> Optional[Path]:
    """The reference source tree the oracle recipe reads: ``$GOSS_REFERENCE``
    when set, else the Makefile's ``REF`` (the recipe is the one place that
    names it); None when that directory does not exist (GPU machines carry
    only the prebuilt ``oracle/_ref``)."""
    env = os.environ.get("GOSS_REFERENCE")
    if env:
        ref = Path(env)
    else:
        try:
            out = subprocess.run(["make", "-s", "--no-print-directory", "-C", str(HERE), "print-ref"],
                                 capture_output=True, text=True, check=True).stdout.strip()
        except (OSError, subprocess.CalledProcessError):
            return None
        if not out:
            return None
        ref = Path(out)
    return ref if (ref / "cpp" / "goss").is_dir() else None


def _cc(name: str) -> str:
    p = Path("/usr/bin") / name
    return str(p) if p.exists() else name


def ref_available() -> bool:
    return (REFDIR / "libgoss_ref_driver.so").exists()


def build_ref_core() -> bool:
    """Build oracle/_ref with the Makefile when the reference sources exist."""
    ref = reference_dir()
    if ref is None:
        return ref_available()
    subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={ref}"], check=True)
    return ref_available()


def build_ref_plugin(variant_dir: Path, force: bool = False) -> Optional[Path]:
    """Compile a variant's goss::ParameterizedODE plugin against the reference headers."""
    variant_dir = Path(variant_dir).resolve()
    out = REFDIR / variant_dir.name / "libplugin.so"
    hdr = variant_dir / "goss_plugin.h"
    if not force and out.exists() and out.stat().st_mtime >= hdr.stat().st_mtime:
        return out
    ref = reference_dir()
    if ref is None or not ref_available():
        return out if out.exists() else None
    out.parent.mkdir(parents=True, exist_ok=True)
    src = out.parent / "plugin.cpp"
    src.write_text(f'#include "{hdr}"\n')
    subprocess.run([_cc("g++"), "-O3", "-DNDEBUG", "-std=c++17", "-fPIC", "-shared", f"-I{ref / 'cpp'}",
                    str(src), f"-L{REFDIR}", "-lgoss_ref", f"-Wl,-rpath,{REFDIR}", "-o", str(out)], check=True)
    return out


def build_ref_plugin_field_states(variant_dir: Path, ode_path: str, field_states) -> Optional[Path]:
    """A variant's plugin generated again with field states (the reference
    fixes them in the plugin class: ParameterizedODE.h:147-150), so that the
    reference's ODESystemSolver::solve returns them.  Generated from the
    reference's .ode file where the sources exist; elsewhere the prebuilt
    library is returned, or None."""
    variant_dir = Path(variant_dir).resolve()
    tag = "_".join(field_states)
    out = REFDIR / f"{variant_dir.name}__fs_{tag}" / "libplugin.so"
    ref = reference_dir()
    if out.exists() and (ref is None or out.stat().st_mtime >= (variant_dir / "model.json").stat().st_mtime):
        return out
    if ref is None or not ref_available():
        return out if out.exists() else None
    import json
    import sys

    sys.path.insert(0, str(HERE.parent))
    from goss_b200.codegen.emit import ModelSource
    from goss_b200.codegen.ir import ModelIR
    from goss_b200.codegen.odeparse import load_ode

    md = json.loads((variant_dir / "model.json").read_text())
    model = load_ode(ref / ode_path)
    ir = ModelIR(model, field_parameters=md["field_parameter_names"], field_states=list(field_states),
                 monitored=md["monitored_names"], linearization=md.get("linearization", "gotran"))
    out.parent.mkdir(parents=True, exist_ok=True)
    hdr = out.parent / "goss_plugin.h"
    hdr.write_text(ModelSource(ir, jacobian=bool(md.get("jacobian"))).emit_goss_plugin())
    src = out.parent / "plugin.cpp"
    src.write_text(f'#include "{hdr}"\n')
    subprocess.run([_cc("g++"), "-O3", "-DNDEBUG", "-std=c++17", "-fPIC", "-shared", f"-I{ref / 'cpp'}",
                    str(src), f"-L{REFDIR}", "-lgoss_ref", f"-Wl,-rpath,{REFDIR}", "-o", str(out)], check=True)
    return out


# plugins built again with field states for the reference's solve():
# (model, .ode path in the reference repository, field states)
FIELD_STATE_PLUGINS = [("tentusscher_panfilov_2006_M_cell", "demo/tentusscher_panfilov_2006_M_cell.ode", ("V", "Ca_i"))]


def field_state_plugin(name: str, field_states) -> Optional[Path]:
    """The prebuilt (or, where the reference sources exist, built now) plugin
    of a FIELD_STATE_PLUGINS entry."""
    import sys

    sys.path.insert(0, str(HERE.parent))
    from goss_b200 import models

    for nm, ode_path, fs in FIELD_STATE_PLUGINS:
        if nm == name and tuple(fs) == tuple(field_states):
            return build_ref_plugin_field_states(models.find_variant(nm), ode_path, fs)
    return None


class RefSystem:
    """The reference's ODESystemSolver over N nodes (implicit: one per node)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            C.CDLL(str(REFDIR / "libgoss_ref.so"), mode=C.RTLD_GLOBAL)
            L = C.CDLL(str(REFDIR / "libgoss_ref_driver.so"))
            L.ref_create.restype = C.c_void_p
            L.ref_create.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(SolverParams), C.c_uint32]
            L.ref_destroy.argtypes = [C.c_void_p]
            L.ref_set_parameter.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
            L.ref_set_states.argtypes = [C.c_void_p, _dp]
            L.ref_get_states.argtypes = [C.c_void_p, _dp]
            L.ref_set_field_parameters.argtypes = [C.c_void_p, _dp]
            L.ref_set_num_threads.argtypes = [C.c_void_p, C.c_uint32]
            L.ref_forward.argtypes = [C.c_void_p, C.c_double, C.c_double]
            L.ref_forward.restype = C.c_int
            L.ref_num_states.argtypes = [C.c_void_p]
            L.ref_last_error.argtypes = [C.c_void_p]
            L.ref_last_error.restype = C.c_char_p
            L.ref_num_jac_comp.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
            L.ref_num_rejected.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
            L.ref_solve.argtypes = [C.c_void_p, _dp, _dp, C.c_uint64, C.c_int]
            L.ref_solve.restype = C.c_int
            L.ref_num_field_states.argtypes = [C.c_void_p]
            L.ref_num_field_states.restype = C.c_uint32
            L.ref_compute_jacobian.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
            L.ref_lu_factorize.argtypes = [C.c_void_p, _dp]
            L.ref_forward_backward_subst.argtypes = [C.c_void_p, _dp, _dp, _dp]
            cls._lib = L
        return cls._lib

    def __init__(self, plugin: Path, class_name: str, solver: str, num_nodes: int, sp: SolverParams):
        L = self.lib()
        self.N = int(num_nodes)
        self.h = L.ref_create(str(plugin).encode(), class_name.encode(), SOLVERS[solver], C.byref(sp), self.N)
        if not self.h:
            raise RuntimeError(f"cannot create reference system from {plugin}")
        self.n = L.ref_num_states(self.h)

    def set_states(self, states: np.ndarray) -> None:
        s = np.ascontiguousarray(states, dtype=np.float64).reshape(self.N, self.n)
        self.lib().ref_set_states(self.h, _ptr(s))

    def get_states(self) -> np.ndarray:
        out = np.zeros((self.N, self.n))
        self.lib().ref_get_states(self.h, _ptr(out))
        return out

    def set_field_parameters(self, fp: np.ndarray) -> None:
        f = np.ascontiguousarray(fp, dtype=np.float64)
        self.lib().ref_set_field_parameters(self.h, _ptr(f))

    def set_parameter(self, name: str, value: float) -> None:
        if self.lib().ref_set_parameter(self.h, name.encode(), float(value)):
            raise RuntimeError(self.lib().ref_last_error(self.h).decode())

    def set_num_threads(self, threads: int) -> None:
        self.lib().ref_set_num_threads(self.h, int(threads))

    def forward(self, t: float, interval: float) -> int:
        return self.lib().ref_forward(self.h, float(t), float(interval))

    def compute_jacobian(self, y: np.ndarray, t: float) -> np.ndarray:
        """The plugin's ODE::compute_jacobian at the default parameters."""
        y = np.array(y, dtype=np.float64)
        jac = np.zeros((self.n, self.n))
        self.lib().ref_compute_jacobian(self.h, _ptr(y), float(t), _ptr(jac))
        return jac

    def lu_factorize(self, mat: np.ndarray) -> None:
        assert mat.dtype == np.float64 and mat.flags.c_contiguous and mat.shape == (self.n, self.n)
        self.lib().ref_lu_factorize(self.h, _ptr(mat))

    def forward_backward_subst(self, mat: np.ndarray, b: np.ndarray) -> np.ndarray:
        x = np.zeros(self.n)
        self.lib().ref_forward_backward_subst(self.h, _ptr(np.ascontiguousarray(mat)),
                                              _ptr(np.ascontiguousarray(b, dtype=np.float64)), _ptr(x))
        return x

    def num_jac_comp(self) -> np.ndarray:
        out = np.zeros(self.N, dtype=np.int64)
        self.lib().ref_num_jac_comp(self.h, out.ctypes.data_as(C.POINTER(C.c_int64)))
        return out

    def solve(self, t: np.ndarray, tangled: bool = True) -> np.ndarray:
        """ODESystemSolver::solve over the times t: [nt][N][nfs] (tangled) or
        [nt][nfs][N]; row 0 is left zero as the reference leaves it."""
        t = np.ascontiguousarray(t, dtype=np.float64)
        nfs = int(self.lib().ref_num_field_states(self.h))
        out = np.zeros((t.size, self.N, nfs) if tangled else (t.size, nfs, self.N))
        if self.lib().ref_solve(self.h, _ptr(out), _ptr(t), t.size, int(tangled)):
            raise RuntimeError(self.lib().ref_last_error(self.h).decode())
        return out

    def num_rejected(self) -> np.ndarray:
        """Rejected steps per node (ESDIRK23a only)."""
        out = np.zeros(self.N, dtype=np.int64)
        if self.lib().ref_num_rejected(self.h, out.ctypes.data_as(C.POINTER(C.c_int64))):
            raise ValueError("num_rejected: the solver keeps no rejection counter")
        return out

    def __del__(self):
        try:
            self.lib().ref_destroy(self.h)
        except Exception:
            pass
