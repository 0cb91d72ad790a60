"""``python -m goss_b200``: the command line of goss (reference
``python/goss/cli.py``) on this package's generator and solvers.

Commands (same names, arguments and options as the reference):

``list-solvers``   the solver table (explicit/implicit, adaptive or not)
``code-params``    the code-generation options and their defaults
``gotran2goss``    ``.ode`` -> the goss C++ plugin header (``--device`` also
                   writes this package's CUDA device model next to it)
``run``            solve one ODE and plot states/monitored values; without
                   matplotlib (or with ``--output``) the series go to a CSV file
"""
from __future__ import annotations

import ast
from pathlib import Path
from typing import Any, Dict, Optional, Sequence

import click
import numpy as np

# GossCodeGeneratorParameters defaults (python/goss/codegeneration.py:163-193)
CODE_PARAM_DEFAULTS: Dict[str, Any] = {
    "state_repr": "named",
    "body_repr": "named",
    "use_cse": False,
    "generate_forward_backward_subst": False,
    "generate_jacobian": False,
    "generate_lu_factorization": False,
    "optimize_exprs": "none",
}


def parse_code_params(text: Optional[str]) -> Dict[str, Any]:
    """``"generate_jacobian=True,use_cse=False"`` -> dict, validated like
    ``ParameterizedODE(code_params=...)`` (the reference's ``CodeParamsType``,
    ``cli.py:37-48``)."""
    from .compilemodule import code_params_jacobian

    if not text:
        return {}
    out: Dict[str, Any] = {}
    for item in text.split(","):
        if not item.strip():
            continue
        if "=" not in item:
            raise click.BadParameter(f"expected key=value, got {item.strip()!r}")
        k, v = (s.strip() for s in item.split("=", 1))
        if v.lower() in ("true", "false"):
            val: Any = v.lower() == "true"
        else:
            try:
                val = ast.literal_eval(v)
            except (ValueError, SyntaxError):
                val = v
        out[k] = val
    try:
        code_params_jacobian(out)
    except (ValueError, TypeError) as exc:
        raise click.BadParameter(str(exc)) from exc
    return out


def _version() -> str:
    from . import __version__

    return __version__


@click.group()
@click.version_option(_version(), prog_name="goss_b200")
def app():
    """goss_b200 - General ODE System Solver on NVIDIA B200.

    Solves gotran .ode models at every node of a mesh on the GPU; the
    commands mirror goss's command line."""


@app.command("list-solvers")
def list_solvers():
    """List available solvers and info about them"""
    from . import solvers

    rows = []
    for name in solvers.GOSSSolvers._member_names_:
        kind = "Explicit" if name in solvers.GOSSExplicitSolvers._member_names_ else "Implicit"
        adapt = "Adaptive" if name in solvers.GOSSAdaptiveSolvers._member_names_ else "Nonadaptive"
        rows.append((name, kind, adapt))
    w = max(len(r[0]) for r in rows)
    click.echo(f"{'Name':>{w}}  Explicit/Implicit  Adaptive/Nonadaptive")
    for name, kind, adapt in rows:
        click.echo(f"{name:>{w}}  {kind:<17}  {adapt}")


@app.command("code-params")
def code_params():
    """List available parameters to codegeneration"""
    for k, v in CODE_PARAM_DEFAULTS.items():
        click.echo(f"{k} = {v}")


def _load(filename: str):
    from .codegen.odeparse import ODEParseError, load_ode

    try:
        return load_ode(filename)
    except ODEParseError as exc:
        raise click.ClickException(str(exc)) from exc


@app.command()
@click.argument("filename", type=click.Path(exists=True, dir_okay=False, resolve_path=True))
@click.option("-o", "--output", default=None, type=click.Path(resolve_path=True), help="Output file name")
@click.option("--field-parameters", "-fp", multiple=True, help="Parameters which should be treated as field parameters")
@click.option("--field-states", "-fs", multiple=True, help="States which should be treated as field states.")
@click.option("--monitored", "-m", multiple=True, help="Monitored intermediates")
@click.option("--list-timings", "-lt", is_flag=True, default=False, help="Print timings of codegeneration.")
@click.option("--code-params", "-cp", default=None, help="Parameters controlling the code generation")
@click.option("--device", is_flag=True, default=False,
              help="Also write the CUDA device model (<output>.cuh) this package compiles")
def gotran2goss(filename, output, field_parameters, field_states, monitored, list_timings, code_params, device):
    """Convert .ode file to goss file"""
    import time

    from .codegen.emit import ModelSource
    from .codegen.ir import ModelIR
    from .compilemodule import code_params_jacobian

    cp = parse_code_params(code_params)
    t0 = time.perf_counter()
    model = _load(filename)
    try:
        ir = ModelIR(model, field_parameters=list(field_parameters), field_states=list(field_states),
                     monitored=list(monitored))
    except ValueError as exc:
        raise click.ClickException(str(exc)) from exc
    src = ModelSource(ir, jacobian=code_params_jacobian(cp))
    out = Path(output).with_suffix(".h") if output else Path(filename).with_suffix(".h")
    out.write_text(src.emit_goss_plugin())
    t1 = time.perf_counter()
    click.echo(f"Output saved to {out}")
    if device:
        cu = out.with_suffix(".cuh")
        cu.write_text(src.emit_device())
        click.echo(f"Device model saved to {cu}")
    if list_timings:
        click.echo(f"code generation: {t1 - t0:.3f} s")


@app.command()
@click.argument("filename", type=click.Path(exists=True, dir_okay=False, resolve_path=True))
@click.option("--end-time", "-T", default=1000.0, type=float, help="End time")
@click.option("--solver", default="ExplicitEuler", help="Which solver to use")
@click.option("--dt", "-dt", default=0.01, type=float, help="Time step")
@click.option("--plot-y", "-y", multiple=True, help="States or monitored to plot on the y axis")
@click.option("--plot-x", "-x", default="time",
              help="Values used for the x axis. Can be time and any valid plot_y variable.")
@click.option("--output", "-o", default=None, type=click.Path(resolve_path=True),
              help="Write x and the plot_y series to this CSV file instead of plotting")
def run(filename, end_time, solver, dt, plot_y, plot_x, output):
    """Solve an ODE"""
    from . import solvers
    from .ode import ParameterizedODE

    if solver not in solvers.GOSSSolvers._member_names_:
        raise click.BadParameter(f"{solver!r} is not one of {', '.join(solvers.GOSSSolvers._member_names_)}",
                                 param_hint="--solver")
    model = _load(filename)
    if not plot_y:
        click.echo("Warning: ploy-y not specified - assume you want to plot 'V'")
        plot_y = ("V",)
    states = list(model.states)
    names = list(model.intermediates)
    for name in list(plot_y) + ([plot_x] if plot_x != "time" else []):
        if name not in states and name not in names:
            raise click.BadParameter(f"{name!r} is neither a state nor an expression of {model.name}")
    monitored = [n for n in plot_y if n in names]
    if plot_x in names and plot_x not in monitored:
        monitored.append(plot_x)
    ode = ParameterizedODE(model, monitored=monitored)
    t = np.arange(0, end_time + dt, dt)
    y = solvers.solver_mapper[solver](ode).solve(t)
    m = ode.monitored_values(y, t) if monitored else None

    def series(name):
        if name == "time":
            return t
        if name in states:
            return y[:, states.index(name)]
        return m[:, monitored.index(name)]

    x = series(plot_x)
    try:
        import matplotlib.pyplot as plt
    except ImportError:
        plt = None
    if output or plt is None:
        out = Path(output) if output else Path(filename).with_suffix(".csv")
        cols = [plot_x] + [n for n in plot_y]
        np.savetxt(out, np.column_stack([x] + [series(n) for n in plot_y]), delimiter=",",
                   header=",".join(cols), comments="")
        click.echo(f"Output saved to {out}")
        return
    for name in plot_y:
        fig, ax = plt.subplots()
        ax.plot(x, series(name))
        ax.set_ylabel(name)
        ax.set_xlabel(plot_x)
    plt.show()


def main(argv: Optional[Sequence[str]] = None) -> int:
    return app.main(args=list(argv) if argv is not None else None, prog_name="goss_b200", standalone_mode=True)
