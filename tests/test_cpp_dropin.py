"""C++ callers of goss's ``ODESystemSolver`` API: ``include/goss_b200.hpp``.

``tests/cpp/dropin_main.cpp`` is written the way a goss C++ user writes a
multi-node solve (``ODESystemSolver(nodes, solver, ode)``, ``forward``,
``solve``, ``set_field_parameters``, solver members such as
``ThetaSolver::theta``; reference ``cpp/goss/ODESystemSolver.h:43-124``).
It is compiled with g++ against the header and ``libgoss_b200.so``; the GPU
cases run it and compare its output with the FP64 oracle.
"""
from __future__ import annotations

import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pyoracle
from helpers import meta, oracle_model, parity, perturbed_states, variant_dir

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "goss_b200" / "_lib"


def _compile(out: Path) -> Path:
    gxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "cpp" / "dropin_main.cpp"), f"-L{LIB}", "-lgoss_b200", "-ldl",
                    f"-Wl,-rpath,{LIB}", "-o", str(out)], check=True, capture_output=True, text=True)
    return out


@pytest.fixture(scope="module")
def dropin(tmp_path_factory):
    import goss_b200  # noqa: F401  (builds/locates the runtime library)
    return _compile(tmp_path_factory.mktemp("cpp") / "dropin_main")


def test_header_compiles_and_links_against_the_runtime(dropin):
    assert dropin.exists()


def _run(exe: Path, vdir: Path, case: str, N: int, arrays, tmp: Path) -> np.ndarray:
    md = meta(vdir)
    lib = vdir / "libgoss_model.so"
    assert lib.exists(), lib
    inp, out = tmp / f"{case}.in", tmp / f"{case}.out"
    np.concatenate([np.ascontiguousarray(a, dtype=np.float64).ravel() for a in arrays]).tofile(inp)
    proc = subprocess.run([str(exe), str(lib), md["variant"], case, str(N), str(inp), str(out)],
                          capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr
    return np.fromfile(out, dtype=np.float64)


@pytest.mark.gpu
def test_cpp_grl1_tp06_1024_nodes_10ms(dropin, tmp_path):
    """The 1,024-node TP06 GRL1 workload (states IC*(1+U(+-5%)), seed 1234),
    10 ms through the C++ classes, within 1e-10 of the oracle."""
    name, N = "tentusscher_panfilov_2006_M_cell", 1024
    vdir = variant_dir(name)
    om = oracle_model(name)
    y0 = perturbed_states(om.ic, N, np.random.default_rng(1234), 0.05)
    gpu = _run(dropin, vdir, "grl1", N, [y0], tmp_path).reshape(N, -1)
    o = pyoracle.OracleSystem(om, "GRL1", N, ldt=0.01)
    o.states[:] = y0
    for k in range(10):
        o.forward(float(k), 1.0)
    assert parity(gpu, o.states, rtol=1e-10) <= 1.0


@pytest.mark.gpu
def test_cpp_field_parameters_and_solve(dropin, tmp_path):
    name, fps = "tentusscher_panfilov_2006_M_cell", ("g_Kr", "g_Ks", "g_CaL", "g_to")
    vdir = variant_dir(name, fps)
    md = meta(vdir)
    om = oracle_model(name, fps)
    N, n, nfp = 100, len(md["state_names"]), len(fps)
    rng = np.random.default_rng(8)
    y0 = perturbed_states(om.ic, N, rng, 0.05)
    defaults = np.array([md["default_parameters"][i] for i in md["field_parameter_indices"]])
    fp = defaults[None, :] * np.exp(0.2 * rng.standard_normal((N, nfp)))
    res = _run(dropin, vdir, "fields", N, [y0, fp], tmp_path)
    states = res[: N * n].reshape(N, n)
    fp_back = res[N * n: N * (n + nfp)].reshape(N, nfp)
    traj = res[N * (n + nfp):].reshape(6, N)
    assert np.array_equal(fp_back, fp)
    o = pyoracle.OracleSystem(om, "GRL1", N, ldt=0.01)
    o.states[:] = y0
    o.field_params[:] = fp
    for k in range(10):
        o.forward(float(k), 1.0)
    iv = md["state_names"].index("V")
    assert np.all(traj[0] == 0.0)  # row 0 is left untouched (ODESystemSolver.cpp:81-99)
    for i in range(1, 6):
        o.forward(9.0 + i, 1.0)
        assert parity(traj[i], o.states[:, iv], rtol=1e-10) <= 1.0
    assert parity(states, o.states, rtol=1e-10) <= 1.0


@pytest.mark.gpu
def test_cpp_theta_solver_tt04(dropin, tmp_path):
    name, N = "tentusscher_2004_mcell", 40
    vdir = variant_dir(name)
    om = oracle_model(name)
    y0 = perturbed_states(om.ic, N, np.random.default_rng(2), 0.02)
    gpu = _run(dropin, vdir, "theta", N, [y0], tmp_path).reshape(N, -1)
    o = pyoracle.OracleSystem(om, "ThetaSolver", N, ldt=0.1, theta=0.5)
    o.states[:] = y0
    for k in range(10):
        assert o.forward(0.1 * k, 0.1) == 0
    assert parity(gpu, o.states, rtol=1e-10) <= 1.0
