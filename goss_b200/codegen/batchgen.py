"""Generate a batch module: several (model variant, explicit solver) kinds in
one persistent kernel (``goss_b200/csrc/goss_batch.cuh``).

The generated ``batch.cu`` includes each variant's ``device.cuh`` (paths
relative to the package directory), a dispatcher from kind index to the
inlined ``explicit_node<Model, T, Solver>``, the per-kind parameter blocks
(parameters + derived constants) and the ``goss_batch_desc`` factory
``goss_b200_batch_<name>()``.
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path
from typing import Dict, List, Sequence, Tuple

from .variant import device_struct

EXPLICIT = {"ExplicitEuler": ("Euler", 0), "RK4": ("RK4", 1), "GRL1": ("GRL1", 2), "GRL2": ("GRL2", 3)}


def batch_name(kinds: Sequence[Tuple[str, str]]) -> str:
    key = json.dumps([list(k) for k in kinds])
    return "batch_" + hashlib.sha1(key.encode()).hexdigest()[:12]


def emit_batch(name: str, kinds: Sequence[Tuple[Path, str]], pkg_dir: Path) -> str:
    """kinds: (variant directory, solver name) per kind."""
    inc, cases, cases_from, sizes, blocks, variants, solvers, nstates, rows = [], [], [], [], [], [], [], [], []
    max_rows = 1
    for k, (vdir, solver) in enumerate(kinds):
        vdir = Path(vdir).resolve()
        md = json.loads((vdir / "model.json").read_text())
        if solver not in EXPLICIT:
            raise ValueError(f"batches run explicit solvers only, got {solver}")
        M = f"goss_b200::models::{device_struct(md['variant'])}"
        rel = vdir.relative_to(Path(pkg_dir).resolve())
        inc.append(f'#include "{rel.as_posix()}/device.cuh"')
        S = f"goss_b200::Explicit::{EXPLICIT[solver][0]}"
        cases.append(f"        case {k}: goss_b200::explicit_node<{M}, T, {S}>(io, node, P, PD); break;")
        cases_from.append(f"        case {k}: goss_b200::explicit_node_from<{M}, T, {S}>(io, node, P, PD, rows, stride); "
                          "break;")
        max_rows = max(max_rows, len(md["state_names"]) + len(md["field_parameter_names"]))
        rows.append(f"        case {k}: *ns = {len(md['state_names'])}; *nf = {len(md['field_parameter_names'])}; return;")
        sizes.append(f"        case {k}: return goss_b200::Dims<{M}>::np;")
        blocks.append(f"        case {k}: {{ double tmp[goss_b200::Dims<{M}>::np]; "
                      f"goss_b200::parameter_block<{M}>(params, tmp); "
                      f"for (int i = 0; i < goss_b200::Dims<{M}>::np; ++i) out[i] = tmp[i]; return; }}")
        variants.append(md["variant"])
        solvers.append(EXPLICIT[solver][1])
        nstates.append(len(md["state_names"]))
    L = [
        f"// Generated by goss_b200.codegen.batchgen (batch {name}); do not edit.",
        "// One persistent kernel for the kinds: " + ", ".join(f"{v}/{s}" for (_, s), v in zip(kinds, variants)),
        '#include "goss_batch.cuh"',
        *inc,
        "",
        "namespace {",
        "struct Dispatch {",
        "    template <typename T>",
        "    __device__ static __forceinline__ void run(int kind, const goss_b200::NodeIO& io, uint32_t node,",
        "                                               const T* __restrict__ P, const double* __restrict__ PD)",
        "    {",
        "        switch (kind) {",
        *cases,
        "        default: break;",
        "        }",
        "    }",
        "    // the same with the node's state rows, then its field-parameter rows, at",
        "    // rows[r * stride] (a tile staged in shared memory)",
        f"    static constexpr int max_rows = {max_rows};",
        "    template <typename T>",
        "    __device__ static __forceinline__ void run_from(int kind, const goss_b200::NodeIO& io, uint32_t node,",
        "                                                    const T* __restrict__ P, const double* __restrict__ PD,",
        "                                                    const double* rows, uint32_t stride)",
        "    {",
        "        switch (kind) {",
        *cases_from,
        "        default: break;",
        "        }",
        "    }",
        "    static int param_block_size(int kind)",
        "    {",
        "        switch (kind) {",
        *sizes,
        "        default: return -1;",
        "        }",
        "    }",
        "    static void row_counts(int kind, uint32_t* ns, uint32_t* nf)",
        "    {",
        "        switch (kind) {",
        *rows,
        "        default: *ns = *nf = 0; return;",
        "        }",
        "    }",
        "    static void param_block(int kind, const double* params, double* out)",
        "    {",
        "        switch (kind) {",
        *blocks,
        "        default: return;",
        "        }",
        "    }",
        "};",
        "static const char* const kind_variants[] = {" + ", ".join(f'"{v}"' for v in variants) + "};",
        "static const int32_t kind_solvers[] = {" + ", ".join(str(s) for s in solvers) + "};",
        "static const uint32_t kind_num_states[] = {" + ", ".join(str(n) for n in nstates) + "};",
        "int launch(const goss_batch_launch* L) { return goss_b200::launch_batch<Dispatch>(L); }",
        "}  // namespace",
        "",
        f'extern "C" GOSS_API const goss_batch_desc* goss_b200_batch_{name}(void)',
        "{",
        f"    static const goss_batch_desc d = {{GOSS_B200_ABI_VERSION, \"{name}\", {len(kinds)}u, kind_variants,",
        "                                      kind_solvers, kind_num_states, launch};",
        "    return &d;",
        "}",
    ]
    return "\n".join(L) + "\n"


def write_batch(name: str, kinds: Sequence[Tuple[Path, str]], outdir: Path, pkg_dir: Path) -> Dict:
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    src = emit_batch(name, kinds, pkg_dir)
    meta = dict(name=name, kinds=[[Path(v).resolve().relative_to(Path(pkg_dir).resolve()).as_posix(), s]
                                  for v, s in kinds])
    for fname, text in (("batch.cu", src), ("batch.json", json.dumps(meta, indent=1) + "\n")):
        p = outdir / fname
        if not p.exists() or p.read_text() != text:
            p.write_text(text)
    return meta
