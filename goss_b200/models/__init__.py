"""Models shipped with goss_b200 as generated, ready-to-build variants.

Each entry of :data:`SHIPPED` is one ``.ode`` model of the reference
repository compiled with one choice of field parameters.  Their generated
sources live in ``goss_b200/models/<variant>/`` (written by
``python -m goss_b200.models.generate`` from the ``.ode`` files) so that the
package builds and runs without the ``.ode`` sources; any other ``.ode`` file
goes through the run-time compiler in :mod:`goss_b200.compilemodule`.
"""
from __future__ import annotations

import json
from pathlib import Path
from typing import Dict, List, Optional, Sequence

HERE = Path(__file__).resolve().parent

# name, path of the .ode file inside the reference repository, field parameters
# (optional: monitored intermediates, jacobian = the analytic Jacobian)
SHIPPED: List[Dict] = [
    dict(name="tentusscher_panfilov_2006_M_cell", ode="demo/tentusscher_panfilov_2006_M_cell.ode",
         field_parameters=[]),
    dict(name="tentusscher_panfilov_2006_M_cell", ode="demo/tentusscher_panfilov_2006_M_cell.ode",
         field_parameters=["g_Kr", "g_Ks", "g_CaL", "g_to"]),
    dict(name="tentusscher_2004_mcell", ode="tests/tentusscher_2004_mcell.ode", field_parameters=[]),
    dict(name="tentusscher_2004_mcell", ode="tests/tentusscher_2004_mcell.ode", field_parameters=["g_Kr", "g_CaL"]),
    dict(name="tentusscher_2004_mcell", ode="tests/tentusscher_2004_mcell.ode", field_parameters=["g_Kr", "g_CaL"],
         jacobian=True),
    dict(name="tentusscher_2004_mcell", ode="tests/tentusscher_2004_mcell.ode",
         field_parameters=["g_Kr", "g_Na", "g_Ks"]),
    dict(name="tentusscher_2004_mcell", ode="tests/tentusscher_2004_mcell.ode",
         field_parameters=["g_Kr", "g_Ks", "g_CaL", "g_to"]),
    dict(name="fitzhughnagumo", ode="tests/fitzhughnagumo.ode", field_parameters=[]),
    dict(name="fitzhughnagumo", ode="tests/fitzhughnagumo.ode", field_parameters=["a", "b"]),
    dict(name="fitzhughnagumo", ode="tests/fitzhughnagumo.ode", field_parameters=[], monitored=["p_42", "p_V"]),
    dict(name="oscilator", ode="tests/oscilator.ode", field_parameters=[]),
    dict(name="oscilator", ode="tests/oscilator.ode", field_parameters=["a", "b"]),
    dict(name="beeler_reuter_1977", ode="cpp/tests/beeler_reuter_1977.ode", field_parameters=[]),
    dict(name="fhn", ode="cpp/tests/fhn.ode", field_parameters=[]),
]


def variant_dirs() -> List[Path]:
    """Directories of all generated shipped variants present in the tree."""
    return sorted(p.parent for p in HERE.glob("*/model.json"))


def find_variant(name: str, field_parameters: Sequence[str] = (), monitored: Sequence[str] = (),
                 linearization: str = "gotran", jacobian: bool = False) -> Optional[Path]:
    """Shipped variant directory for a model name and code-generation choice."""
    for vdir in variant_dirs():
        md = json.loads((vdir / "model.json").read_text())
        if (md["name"] == name and md["field_parameter_names"] == list(field_parameters)
                and md["monitored_names"] == list(monitored) and md.get("linearization", "gotran") == linearization
                and bool(md.get("jacobian", False)) == bool(jacobian)):
            return vdir
    return None


def shipped_names() -> List[str]:
    return sorted({json.loads((d / "model.json").read_text())["name"] for d in variant_dirs()})
