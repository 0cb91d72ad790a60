"""Compile and load model variants (replacement of goss's cppyy JIT).

The reference turns a gotran ODE into C++ with ``GossCodeGenerator`` and
JIT-compiles it with cppyy (``python/goss/compilemodule.py:20-117``).  Here a
model becomes a *variant*: generated CUDA sources compiled by nvcc for sm_100a
into ``libgoss_model.so``, whose ``goss_b200_model_<variant>()`` factory
returns the ``goss_model_desc`` the runtime drives.

Shipped variants live in ``goss_b200/models/``; any other model/choice is
generated and compiled into the in-tree cache ``goss_b200/_jit/``.
"""
from __future__ import annotations

import ctypes as C
import json
import threading
from pathlib import Path
from typing import Dict, Optional, Sequence, Union

from . import _capi
from .build import build_variant
from .codegen.odeparse import ODEModel, load_ode
from .codegen.variant import model_hash, variant_id, write_variant

PKG = Path(__file__).resolve().parent
JIT_DIR = PKG / "_jit"

_lock = threading.Lock()
_loaded: Dict[str, "ModelModule"] = {}


class ModelModule:
    """A compiled model variant: metadata plus the loaded CUDA module."""

    def __init__(self, vdir: Path):
        self.dir = Path(vdir)
        self.meta = json.loads((self.dir / "model.json").read_text())
        self.variant = self.meta["variant"]
        so = build_variant(self.dir)
        self._lib = C.CDLL(str(so))
        factory = getattr(self._lib, f"goss_b200_model_{self.variant}")
        factory.restype = C.POINTER(_capi.ModelDesc)
        self.desc = factory()
        if not self.desc or self.desc.contents.abi_version != _capi.ABI_VERSION:
            raise _capi.ExtensionMissingError(f"{so}: model descriptor has the wrong ABI version")
        _capi.lib()  # the runtime must be loadable as well

    # metadata shortcuts
    @property
    def name(self) -> str:
        return self.meta["name"]

    @property
    def num_states(self) -> int:
        return len(self.meta["state_names"])

    def __repr__(self) -> str:
        return f"ModelModule({self.variant})"


def load_variant(vdir: Union[str, Path]) -> ModelModule:
    vdir = Path(vdir).resolve()
    key = str(vdir)
    with _lock:
        mod = _loaded.get(key)
        if mod is None:
            mod = ModelModule(vdir)
            _loaded[key] = mod
        return mod


# GossCodeGeneratorParameters (python/goss/codegeneration.py:163-193): option
# -> allowed values (None: a bool).  Unknown keys are ignored, as the
# reference's pydantic model ignores them.
_CODE_PARAMS = {
    "state_repr": ("named", "array"),
    "body_repr": ("named", "array", "reused_array"),
    "use_cse": None,
    "generate_forward_backward_subst": None,
    "generate_jacobian": None,
    "generate_lu_factorization": None,
    "optimize_exprs": ("none", "numerals", "numerals_symbols"),
}


def code_params_jacobian(code_params: Optional[dict]) -> bool:
    """Validate the reference's ``code_params`` and return whether the analytic
    Jacobian is generated.

    Only ``generate_jacobian`` changes the compiled model.  The representation
    and CSE options shape the reference's C++ text, not its values; the
    generated LU factorisation and substitution
    (``generate_lu_factorization``, ``generate_forward_backward_subst``) are
    what the implicit kernels always run: structure-aware Doolittle LU and
    substitution, which equal the dense ones bit for bit on finite matrices.
    """
    if code_params is None:
        return False
    if not isinstance(code_params, dict):
        raise TypeError("code_params must be a dict")
    for key, allowed in _CODE_PARAMS.items():
        if key not in code_params:
            continue
        v = code_params[key]
        v = getattr(v, "value", v)  # enum members
        if allowed is None:
            if not isinstance(v, (bool, int)) or isinstance(v, int) and v not in (0, 1):
                raise ValueError(f"code_params[{key!r}] must be a bool, got {v!r}")
        elif v not in allowed:
            raise ValueError(f"code_params[{key!r}] must be one of {'|'.join(allowed)}, got {v!r}")
    return bool(code_params.get("generate_jacobian", False))


def jit(model: Union[ODEModel, str, Path], field_parameters: Sequence[str] = (), monitored: Sequence[str] = (),
        linearization: str = "gotran", code_params: Optional[dict] = None) -> ModelModule:
    """Compiled variant of ``model`` with the given field parameters.

    ``model`` is a parsed :class:`ODEModel`, a path to a ``.ode`` file or the
    name of a shipped model; ``code_params`` are the reference generator's
    options (``compilemodule.py:85-117``), see :func:`code_params_jacobian`.
    """
    from . import models

    jacobian = code_params_jacobian(code_params)
    if isinstance(model, (str, Path)) and not Path(model).suffix and not Path(model).with_suffix(".ode").is_file():
        vdir = models.find_variant(str(model), field_parameters, monitored, linearization, jacobian)
        if vdir is None:
            raise FileNotFoundError(
                f"'{model}' is neither a .ode file nor a shipped model variant with field parameters "
                f"{list(field_parameters)} and monitored {list(monitored)}; shipped models: {models.shipped_names()}")
        return load_variant(vdir)
    if isinstance(model, (str, Path)):
        model = load_ode(model)
    h = model_hash(model, field_parameters, monitored, linearization, jacobian)
    vdir = models.find_variant(model.name, field_parameters, monitored, linearization, jacobian)
    if vdir is not None and json.loads((vdir / "model.json").read_text()).get("hash") == h:
        return load_variant(vdir)
    ident = variant_id(model, field_parameters, monitored, linearization, jacobian)
    ident = f"{ident}__{h[:10]}" if "__" not in ident else f"{ident}_{h[:10]}"
    vdir = JIT_DIR / ident
    with _lock:
        if not (vdir / "model.json").exists() or json.loads((vdir / "model.json").read_text()).get("hash") != h:
            write_variant(model, vdir, field_parameters=field_parameters, monitored=monitored,
                          linearization=linearization, ident=ident, jacobian=jacobian)
    return load_variant(vdir)
