"""Build the native parts in-tree with nvcc (sm_100a).

* ``goss_b200/_lib/libgoss_b200.so``: the runtime behind ``include/goss_b200.h``.
* ``<variant>/libgoss_model.so``: the solver kernels of one model variant
  (``goss_b200/models/<variant>/`` for the shipped models, the JIT cache
  ``goss_b200/_jit/<variant>/`` for models compiled at run time).

Builds are incremental: a target is rebuilt when any of its sources is newer.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path
from typing import Iterable, List, Optional

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIBDIR = PKG / "_lib"
RUNTIME_SO = LIBDIR / "libgoss_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc() -> str:
    exe = shutil.which("nvcc")
    if exe:
        return exe
    cand = Path("/usr/local/cuda/bin/nvcc")
    if cand.exists():
        return str(cand)
    raise RuntimeError("nvcc not found: the goss_b200 CUDA extensions cannot be built")


def _digest(deps: Iterable[Path], flags: Iterable[str] = ()) -> str:
    h = hashlib.sha1()
    for d in deps:
        h.update(str(d.name).encode())
        h.update(d.read_bytes() if d.exists() else b"<missing>")
    h.update(" ".join(flags).encode())
    return h.hexdigest()


def _stale(target: Path, deps: Iterable[Path], flags: Iterable[str] = ()) -> bool:
    """A target is stale when it is missing or its sources' content changed
    (content hashes, not mtimes, so copies of the tree do not rebuild)."""
    stamp = target.with_name(target.name + ".sha1")
    if not target.exists() or not stamp.exists():
        return True
    return stamp.read_text().strip() != _digest(deps, flags)


def _stamp(target: Path, deps: Iterable[Path], flags: Iterable[str] = ()) -> None:
    target.with_name(target.name + ".sha1").write_text(_digest(deps, flags) + "\n")


def _run(cmd: List[str], cwd: Optional[Path] = None) -> None:
    proc = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")


def build_runtime(force: bool = False) -> Path:
    src = CSRC / "runtime.cu"
    deps = [src, INCLUDE / "goss_b200.h"]
    if force or _stale(RUNTIME_SO, deps):
        LIBDIR.mkdir(parents=True, exist_ok=True)
        tmp = RUNTIME_SO.with_suffix(".so.tmp")
        _run([nvcc(), *ARCH, *COMMON, "-shared", str(src), "-o", str(tmp)])
        os.replace(tmp, RUNTIME_SO)
        _stamp(RUNTIME_SO, deps)
    return RUNTIME_SO


def variant_deps(vdir: Path) -> List[Path]:
    return [vdir / "module.cu", vdir / "device.cuh", CSRC / "goss_kernels.cuh", CSRC / "goss_device_math.cuh",
            CSRC / "goss_adjoint.cuh", INCLUDE / "goss_b200.h"]


def build_variant(vdir: Path, force: bool = False, extra_flags: Optional[List[str]] = None) -> Path:
    """Compile one variant directory into ``libgoss_model.so``."""
    vdir = Path(vdir)
    out = vdir / "libgoss_model.so"
    flags = ["--use_fast_math"] + (extra_flags or [])
    if force or _stale(out, variant_deps(vdir), flags):
        tmp = out.with_suffix(f".so.{os.getpid()}.tmp")
        _run([nvcc(), *ARCH, *COMMON, *flags, f"-I{vdir}", "-shared", str(vdir / "module.cu"), "-o", str(tmp)])
        os.replace(tmp, out)
        _stamp(out, variant_deps(vdir), flags)
    return out


def batch_deps(bdir: Path) -> List[Path]:
    import json

    meta = json.loads((Path(bdir) / "batch.json").read_text())
    deps = [Path(bdir) / "batch.cu", CSRC / "goss_batch.cuh", CSRC / "goss_kernels.cuh",
            CSRC / "goss_device_math.cuh", INCLUDE / "goss_b200.h"]
    deps += [PKG / v / "device.cuh" for v, _ in meta["kinds"]]
    return deps


def build_batch(bdir: Path, force: bool = False) -> Path:
    """Compile one batch module directory into ``libgoss_batch.so``."""
    bdir = Path(bdir)
    out = bdir / "libgoss_batch.so"
    flags = ["--use_fast_math"]
    if force or _stale(out, batch_deps(bdir), flags):
        tmp = out.with_suffix(f".so.{os.getpid()}.tmp")
        _run([nvcc(), *ARCH, *COMMON, *flags, f"-I{PKG}", "-shared", str(bdir / "batch.cu"), "-o", str(tmp)])
        os.replace(tmp, out)
        _stamp(out, batch_deps(bdir), flags)
    return out


def build_all(variant_dirs: Iterable[Path], force: bool = False, jobs: Optional[int] = None,
              batch_dirs: Iterable[Path] = ()) -> List[Path]:
    """Runtime plus every variant and batch module, compiled in parallel."""
    build_runtime(force)
    jobs_list = [(build_variant, d) for d in variant_dirs] + [(build_batch, d) for d in batch_dirs]
    jobs = jobs or max(1, min(len(jobs_list), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        return list(ex.map(lambda fd: fd[0](fd[1], force), jobs_list))
