"""Generate the golden vectors that pin the model code generator.

Run from the repository root in a checkout that has the reference sources
at ``$GOSS_REFERENCE`` (or where the oracle recipe ``oracle/Makefile`` reads
them, ``make -s -C oracle print-ref``)::

    GOSS_REFERENCE=/path/to/goss python tests/golden/make_golden.py

Sources of truth (all from the reference repository, used read-only):

* ``cpp/tests/fhn.h``, ``cpp/tests/beeler_reuter_1977.h``, ``tests/oscilator.h``:
  gotran-generated goss model classes.  A small C++ driver (written here,
  compiled into a temporary directory together with the reference's
  ``cpp/goss/ODE.cpp``) evaluates their ``eval`` and ``linearized_eval`` at
  seeded random states.
* ``benchmarks/tentusscher_panfilov_2006_M_cell.py``: the gotran-generated
  numpy right-hand side of the TP06 M-cell model.  Its ``rhs`` function and
  the parameter vector of ``main()`` are extracted with :mod:`ast` and
  evaluated at seeded random states.

Outputs ``tests/golden/*.npz``; the tests compare the project's generated
code against them and never read the reference at test time.
"""
from __future__ import annotations

import ast
import math
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1] / "oracle"))
import pyoracle  # noqa: E402

_ref = pyoracle.reference_dir()
if _ref is None:
    sys.exit("make_golden.py: the reference sources were not found; set GOSS_REFERENCE to a goss checkout")
REF = _ref

CPP_FIXTURES = [
    # (model name, header relative to REF, class name, .ode relative to REF)
    ("fhn", "cpp/tests/fhn.h", "Fhn", "cpp/tests/fhn.ode"),
    ("beeler_reuter_1977", "cpp/tests/beeler_reuter_1977.h", "Beeler_reuter_1977",
     "cpp/tests/beeler_reuter_1977.ode"),
    ("oscilator", "tests/oscilator.h", "Oscilator", "tests/oscilator.ode"),
]

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <string>
#define DLL_EXPORT
#include "%(header)s"

// reads: nsamples, then per sample [time, states...]; writes per sample
// eval values, linearized rhs, linearized linear, and the default params
int main(int argc, char** argv)
{
    goss::%(cls)s ode;
    const unsigned n = ode.num_states();
    FILE* in = std::fopen(argv[1], "rb");
    FILE* out = std::fopen(argv[2], "wb");
    int ns = 0;
    if (std::fread(&ns, sizeof(int), 1, in) != 1) return 1;
    std::vector<double> y(n), v(n), lin(n), rhs(n);
    for (int s = 0; s < ns; ++s) {
        double t;
        if (std::fread(&t, sizeof(double), 1, in) != 1) return 1;
        if (std::fread(y.data(), sizeof(double), n, in) != n) return 1;
        ode.eval(y.data(), t, v.data());
        for (unsigned i = 0; i < n; ++i) lin[i] = 0.0;
        ode.linearized_eval(y.data(), t, lin.data(), rhs.data(), false);
        std::fwrite(v.data(), sizeof(double), n, out);
        std::fwrite(rhs.data(), sizeof(double), n, out);
        std::fwrite(lin.data(), sizeof(double), n, out);
    }
    const auto& pn = ode.get_parameter_names();
    for (const auto& name : pn) {
        double p = ode.get_parameter(name);
        std::fwrite(&p, sizeof(double), 1, out);
    }
    std::vector<unsigned char> lt(n);
    for (unsigned i = 0; i < n; ++i) lt[i] = ode.linear_term(i);
    std::fwrite(lt.data(), 1, n, out);
    std::fclose(out);
    return 0;
}
"""


def sample_states(ic: np.ndarray, rng: np.random.Generator, ns: int) -> np.ndarray:
    """States around the initial condition; zero entries get small values."""
    ic = np.asarray(ic, dtype=np.float64)
    scale = np.where(ic != 0.0, np.abs(ic), 0.1)
    u = rng.uniform(-0.3, 0.3, size=(ns, ic.size))
    return ic + scale * u


def cpp_fixture(name, header, cls, ode_rel, rng, ns=64):
    sys.path.insert(0, str(HERE.parents[1]))
    from goss_b200.codegen.odeparse import load_ode

    model = load_ode(REF / ode_rel)
    ic = np.array(list(model.states.values()))
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        (td / "driver.cpp").write_text(DRIVER % dict(header=str(REF / header), cls=cls))
        exe = td / "driver"
        subprocess.run(["g++", "-O2", "-std=c++17", f"-I{REF / 'cpp'}", str(td / "driver.cpp"),
                        str(REF / "cpp/goss/ODE.cpp"), "-o", str(exe)], check=True)
        states = sample_states(ic, rng, ns)
        times = rng.uniform(0.0, 3.0, size=ns)
        with open(td / "in.bin", "wb") as f:
            f.write(np.int32(ns).tobytes())
            for t, y in zip(times, states):
                f.write(np.float64(t).tobytes())
                f.write(y.astype(np.float64).tobytes())
        subprocess.run([str(exe), str(td / "in.bin"), str(td / "out.bin")], check=True)
        raw = (td / "out.bin").read_bytes()
    n = ic.size
    body = np.frombuffer(raw[: ns * 3 * n * 8], dtype=np.float64).reshape(ns, 3, n)
    npar = len(model.parameters)
    params = np.frombuffer(raw[ns * 3 * n * 8: ns * 3 * n * 8 + npar * 8], dtype=np.float64)
    lt = np.frombuffer(raw[ns * 3 * n * 8 + npar * 8:], dtype=np.uint8)
    np.savez(HERE / f"{name}_cpp_fixture.npz", times=times, states=states, eval=body[:, 0],
             lin_rhs=body[:, 1], linear=body[:, 2], params=params, linear_terms=lt,
             source=np.array(f"{header} ({cls})"))
    print(f"{name}: {ns} samples, {n} states, {npar} params")


def tp06_numpy_fixture(rng, ns=64):
    path = REF / "benchmarks/tentusscher_panfilov_2006_M_cell.py"
    tree = ast.parse(path.read_text())
    rhs_def = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "rhs")
    main_def = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "main")
    params = None
    for st in ast.walk(main_def):
        if isinstance(st, ast.Assign) and isinstance(st.targets[0], ast.Name) and st.targets[0].id == "init_parameters":
            params = np.array(ast.literal_eval(st.value.args[0]), dtype=np.float64)
    assert params is not None
    ns_ = {"math": math, "np": np}
    np.float_ = np.float64  # the fixture targets numpy<2
    exec(compile(ast.Module(body=[rhs_def], type_ignores=[]), str(path), "exec"), ns_)
    rhs = ns_["rhs"]
    unpack = [st for st in rhs_def.body if isinstance(st, ast.Assign) and isinstance(st.targets[0], ast.Tuple)]
    state_order = [e.id for e in unpack[0].targets[0].elts]
    param_order = [e.id for e in unpack[1].targets[0].elts]
    sys.path.insert(0, str(HERE.parents[1]))
    from goss_b200.codegen.odeparse import load_ode

    model = load_ode(REF / "demo/tentusscher_panfilov_2006_M_cell.ode")
    ic = np.array([model.states[s] for s in state_order])
    states = sample_states(ic, rng, ns)
    # keep V in the physiological range and include both branches of the
    # V < -40 conditionals
    states[:, state_order.index("V")] = rng.uniform(-90.0, 40.0, size=ns)
    times = rng.uniform(0.0, 20.0, size=ns)
    values = np.array([rhs(t, y, params) for t, y in zip(times, states)])
    np.savez(HERE / "tp06_numpy_fixture.npz", times=times, states=states, values=values, params=params,
             state_order=np.array(state_order), param_order=np.array(param_order),
             source=np.array("benchmarks/tentusscher_panfilov_2006_M_cell.py rhs()"))
    print(f"tp06 numpy rhs: {ns} samples")


def main():
    if not REF.is_dir():
        raise SystemExit(f"reference sources not found at {REF}")
    rng = np.random.default_rng(20260314)
    for args in CPP_FIXTURES:
        cpp_fixture(*args, rng=rng)
    tp06_numpy_fixture(rng)


if __name__ == "__main__":
    main()
