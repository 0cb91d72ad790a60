"""``python -m goss_b200``: the reference's command line (``python/goss/cli.py``)."""
from __future__ import annotations

import numpy as np
import pytest
from click.testing import CliRunner

import pyoracle
from goss_b200.cli import app, parse_code_params
from helpers import oracle_model


def _ode_file(tmp_path, name="oscilator"):
    """A .ode file for the CLI: the shipped oscillator restated (the reference's
    tests/oscilator.ode: x' = -a*y, y' = b*x, monitored energy)."""
    p = tmp_path / f"{name}.ode"
    p.write_text(
        'states(x=1.0, y=0.0)\n'
        'parameters(a=1.0, b=1.0)\n'
        'energy = a*y + b*x\n'
        'dx_dt = -a*y\n'
        'dy_dt = b*x\n')
    return p


def test_list_solvers():
    r = CliRunner().invoke(app, ["list-solvers"])
    assert r.exit_code == 0, r.output
    lines = r.output.splitlines()
    assert any("ESDIRK23a" in l and "Implicit" in l and "Adaptive" in l for l in lines)
    assert any("GRL1" in l and "Explicit" in l and "Nonadaptive" in l for l in lines)
    assert sum(1 for l in lines[1:] if l.strip()) == 10


def test_code_params_lists_defaults():
    r = CliRunner().invoke(app, ["code-params"])
    assert r.exit_code == 0
    assert "generate_jacobian = False" in r.output and "optimize_exprs = none" in r.output


def test_parse_code_params():
    assert parse_code_params("generate_jacobian=True, use_cse=false,optimize_exprs=numerals") == {
        "generate_jacobian": True, "use_cse": False, "optimize_exprs": "numerals"}
    assert parse_code_params(None) == {}
    import click

    with pytest.raises(click.BadParameter):
        parse_code_params("body_repr=tree")
    with pytest.raises(click.BadParameter):
        parse_code_params("generate_jacobian")


def test_gotran2goss_writes_plugin_with_jacobian(tmp_path):
    ode = _ode_file(tmp_path)
    out = tmp_path / "gen" / "osc"
    out.parent.mkdir()
    r = CliRunner().invoke(app, ["gotran2goss", str(ode), "-o", str(out), "-fp", "a", "-fs", "x", "-m", "energy",
                                 "-cp", "generate_jacobian=True,generate_lu_factorization=True", "--device"])
    assert r.exit_code == 0, r.output
    h = (tmp_path / "gen" / "osc.h").read_text()
    # the reference's test_GossCodeGenerator checks (tests/test_codegeneration.py:26-32)
    assert "#include \"goss/ParameterizedODE.h\"" in h
    assert "void compute_jacobian" in h and "void linearized_eval" in h
    assert "monitored[0] = " in h and "create_Oscilator" in h
    assert "has_jacobian = true" in (tmp_path / "gen" / "osc.cuh").read_text()
    r = CliRunner().invoke(app, ["gotran2goss", str(ode), "-o", str(tmp_path / "plain")])
    assert r.exit_code == 0 and "compute_jacobian" not in (tmp_path / "plain.h").read_text()


def test_gotran2goss_rejects_unknown_names(tmp_path):
    ode = _ode_file(tmp_path)
    r = CliRunner().invoke(app, ["gotran2goss", str(ode), "-fp", "not_a_parameter"])
    assert r.exit_code != 0 and "not_a_parameter" in r.output


@pytest.mark.gpu
def test_run_writes_series(tmp_path):
    ode = _ode_file(tmp_path)
    csv = tmp_path / "out.csv"
    r = CliRunner().invoke(app, ["run", str(ode), "-T", "1.0", "-dt", "0.1", "--solver", "RK4", "-y", "x",
                                 "-y", "energy", "-o", str(csv)])
    assert r.exit_code == 0, r.output
    data = np.loadtxt(csv, delimiter=",", skiprows=1)
    assert data.shape == (11, 3)
    om = oracle_model("oscilator")
    o = pyoracle.OracleSystem(om, "RK4", 1, ldt=0.1)
    xs = [1.0]
    for k in range(10):
        o.forward(0.1 * k, 0.1)
        xs.append(float(o.states[0, 0]))
    assert np.allclose(data[:, 0], np.arange(11) * 0.1)
    assert np.allclose(data[:, 1], xs, rtol=1e-12, atol=1e-14)
