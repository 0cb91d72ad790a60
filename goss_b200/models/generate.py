"""Regenerate the shipped model variants from the reference ``.ode`` files.

Usage (needs the reference sources, default ``/root/reference``)::

    GOSS_REFERENCE=/path/to/goss python -m goss_b200.models.generate
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

from ..codegen.odeparse import load_ode
from ..codegen.variant import variant_id, write_variant
from . import HERE, SHIPPED


def main() -> int:
    ref = Path(os.environ.get("GOSS_REFERENCE", "/root/reference"))
    if not ref.is_dir():
        print(f"reference sources not found at {ref}", file=sys.stderr)
        return 1
    for entry in SHIPPED:
        model = load_ode(ref / entry["ode"])
        assert model.name == entry["name"], (model.name, entry["name"])
        mon = entry.get("monitored", [])
        ident = variant_id(model, entry["field_parameters"], mon)
        md = write_variant(model, HERE / ident, field_parameters=entry["field_parameters"], monitored=mon)
        print(f"{ident}: {len(md['state_names'])} states, {len(md['parameter_names'])} parameters, "
              f"field parameters {md['field_parameter_names']}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
