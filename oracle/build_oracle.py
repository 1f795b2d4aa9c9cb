"""Build recipe for the test oracles -- TEST INFRASTRUCTURE ONLY.

* ``oracle/liboracle.so``: the CPU restatement (``cpu_oracle.cpp``), g++.
* ``oracle/_ref/libtfgref.so``: the reference's own kernels, compiled for
  sm_100a straight from the reference checkout (``RenderKernel.cu`` and
  ``NrcKernel.cu`` where they lie, unmodified) together with
  ``ref_shim.cu``.  Only built when the reference checkout is present (it is
  absent on the GPU machines, which use the prebuilt file).  The reference's
  own build (CMake, tiny-cuda-nn, tinybvh, GLFW, assimp) is not used: these two
  files need none of it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent


def reference_dir() -> Path | None:
    """The reference checkout: ``TFG_REFERENCE_DIR``, else a checkout named
    ``reference`` beside the repository; None when neither holds the kernel
    sources (the prebuilt library is used then)."""
    for d in (os.environ.get("TFG_REFERENCE_DIR"), str(ROOT.parent / "reference")):
        if d and (Path(d) / "RenderKernel.cu").exists():
            return Path(d)
    return None


ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libtfgref.so"


def _newer(target: Path, deps: list[Path]) -> bool:
    return target.exists() and all(target.stat().st_mtime >= d.stat().st_mtime for d in deps if d.exists())


def build_cpu(force: bool = False) -> Path:
    src = HERE / "cpu_oracle.cpp"
    deps = [src, ROOT / "include" / "tfg_pt.h"]
    if not force and _newer(ORACLE_LIB, deps):
        return ORACLE_LIB
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-std=c++17", "-fPIC", "-shared", "-pthread",
           "-I", str(ROOT / "include"), str(src), "-o", str(ORACLE_LIB)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stderr}")
    return ORACLE_LIB


def build_ref(force: bool = False) -> Path | None:
    """Compile the reference kernels; without the checkout the prebuilt
    library is returned (None when there is none)."""
    ref_dir = reference_dir()
    if ref_dir is None:
        return REF_LIB if REF_LIB.exists() else None
    srcs = [ref_dir / "RenderKernel.cu", ref_dir / "NrcKernel.cu"]
    shim = HERE / "ref_shim.cu"
    headers = sorted(ref_dir.glob("*.h")) + sorted(ref_dir.glob("*.cuh"))
    if not force and _newer(REF_LIB, [shim, *srcs, *headers]):
        return REF_LIB
    nvcc = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    REF_LIB.parent.mkdir(exist_ok=True)
    cmd = [nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
           "-shared", "-w", "-I", str(ref_dir), *map(str, srcs), str(shim), "-o", str(REF_LIB)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"reference kernel build failed:\n{res.stderr}")
    return REF_LIB


def build(force: bool = False) -> None:
    build_cpu(force)
    build_ref(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(ORACLE_LIB, REF_LIB if REF_LIB.exists() else "(no reference build)")
