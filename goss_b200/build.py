"""Build the native parts in-tree with nvcc (sm_100a).

* ``goss_b200/_lib/libgoss_b200.so``: the runtime behind ``include/goss_b200.h``.
* ``<variant>/libgoss_model.so``: the solver kernels of one model variant
  (``goss_b200/models/<variant>/`` for the shipped models, the JIT cache
  ``goss_b200/_jit/<variant>/`` for models compiled at run time).

Builds are incremental: a target is rebuilt when any of its sources is newer.
"""
from __future__ import annotations

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


def _stale(target: Path, deps: Iterable[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


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
    return RUNTIME_SO


def variant_deps(vdir: Path) -> List[Path]:
    return [vdir / "module.cu", vdir / "device.cuh", CSRC / "goss_kernels.cuh", CSRC / "goss_device_math.cuh",
            INCLUDE / "goss_b200.h"]


def build_variant(vdir: Path, force: bool = False, extra_flags: Optional[List[str]] = None) -> Path:
    """Compile one variant directory into ``libgoss_model.so``."""
    vdir = Path(vdir)
    out = vdir / "libgoss_model.so"
    if force or _stale(out, variant_deps(vdir)):
        tmp = out.with_suffix(f".so.{os.getpid()}.tmp")
        flags = ["--use_fast_math", f"-I{vdir}"] + (extra_flags or [])
        _run([nvcc(), *ARCH, *COMMON, *flags, "-shared", str(vdir / "module.cu"), "-o", str(tmp)])
        os.replace(tmp, out)
    return out


def build_all(variant_dirs: Iterable[Path], force: bool = False, jobs: Optional[int] = None) -> List[Path]:
    """Runtime plus every variant, variants compiled in parallel."""
    build_runtime(force)
    dirs = list(variant_dirs)
    jobs = jobs or max(1, min(len(dirs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        return list(ex.map(lambda d: build_variant(d, force), dirs))
