"""Build recipe for the reference-side binding ``tfg_b200/dropin/libtfgdropin.so``.

``reference_wrappers.cu`` implements the reference's host entry points
(RenderKernel.h, NrcKernel.h, class TinyBVH of tinybvh_wrapper.h, class
ColorMLP of the replacement mlp.h beside it) over libtfgpt's C ABI.  It is
compiled against the reference's own, unmodified headers -- found through
``TFG_REFERENCE_DIR`` or a ``reference`` checkout beside the repository -- and
linked to ``tfg_b200/libtfgpt.so``.  Without the headers the prebuilt library
(if any) is kept.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
SRC = HERE / "reference_wrappers.cu"
LIB = HERE / "libtfgdropin.so"


def reference_dir() -> Path | None:
    """``TFG_REFERENCE_DIR``, else a checkout named ``reference`` beside the
    repository; None when neither holds the reference's headers."""
    for d in (os.environ.get("TFG_REFERENCE_DIR"), str(ROOT.parent / "reference")):
        if d and (Path(d) / "RenderKernel.h").exists():
            return Path(d)
    return None


def build(force: bool = False) -> Path | None:
    ref = reference_dir()
    if ref is None:
        return LIB if LIB.exists() else None
    core = PKG / "libtfgpt.so"
    deps = [SRC, HERE / "mlp.h", ROOT / "include" / "tfg_pt.h", core] + sorted(ref.glob("*.h"))
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in deps if d.exists()):
        return LIB
    nvcc = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
           "-shared", "-w", "-I", str(HERE), "-I", str(ROOT / "include"), "-I", str(ref), str(SRC), "-o", str(LIB),
           "-L", str(PKG), "-ltfgpt", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/.."]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"reference binding build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
