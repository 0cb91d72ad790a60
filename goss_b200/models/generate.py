"""Regenerate the shipped model variants from the reference ``.ode`` files.

Usage (needs the reference sources; there is no default location)::

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
    env = os.environ.get("GOSS_REFERENCE")
    if not env:
        print("GOSS_REFERENCE is not set: point it at a goss checkout (the .ode files are read from it)",
              file=sys.stderr)
        return 1
    ref = Path(env)
    if not ref.is_dir():
        print(f"reference sources not found at {ref} (GOSS_REFERENCE)", file=sys.stderr)
        return 1
    for entry in SHIPPED:
        model = load_ode(ref / entry["ode"])
        assert model.name == entry["name"], (model.name, entry["name"])
        mon = entry.get("monitored", [])
        jac = entry.get("jacobian", False)
        ident = variant_id(model, entry["field_parameters"], mon, jacobian=jac)
        md = write_variant(model, HERE / ident, field_parameters=entry["field_parameters"], monitored=mon,
                           jacobian=jac)
        print(f"{ident}: {len(md['state_names'])} states, {len(md['parameter_names'])} parameters, "
              f"field parameters {md['field_parameter_names']}")
    # batch modules over shipped variants
    from ..batches import HERE as BATCHES, SHIPPED_BATCHES
    from ..codegen.batchgen import write_batch
    from . import find_variant

    pkg = HERE.parent
    for b in SHIPPED_BATCHES:
        kinds = []
        for name, fps, solver in b["kinds"]:
            vdir = find_variant(name, fps)
            assert vdir is not None, (name, fps)
            kinds.append((vdir, solver))
        write_batch(b["name"], kinds, BATCHES / b["name"], pkg)
        print(f"batch {b['name']}: {[(k[0].name, k[1]) for k in kinds]}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
