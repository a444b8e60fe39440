"""Build ``libhexdyn.so`` (sm_100a) in-tree with nvcc.

The dycore kernels are compiled twice from the same source: the strict build
(``-fmad=false``: every FP32 operation rounded on its own, bit-identical to the
reference's NumPy authority) and the fast build (``-fmad=true``).  The C ABI
layer is compiled strict.  Objects go to ``csrc/_build/``; the library lands
next to this file so that it travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
CSRC = PACKAGE_DIR.parent / "csrc"
INCLUDE = PACKAGE_DIR.parent.parent / "include"
LIBRARY = PACKAGE_DIR / "libhexdyn.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-ftz=false", "-prec-div=true", "-prec-sqrt=true", "-I", str(CSRC), "-I", str(INCLUDE)]
UNITS = {
    "kernels_strict.cu": ["-fmad=false"],
    "kernels_fast.cu": ["-fmad=true"],
    "hexdyn_abi.cu": ["-fmad=false"],
    "mlp_umma.cu": [],
}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the hexdyn CUDA library cannot be built")
    return path


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
                  + list(INCLUDE.glob("*.h")))


def needs_build() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    return any(p.stat().st_mtime > built for p in _sources())


def build_library(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compile and link the library; returns its path."""
    if not force and not needs_build():
        return LIBRARY
    out_dir = CSRC / "_build"
    out_dir.mkdir(exist_ok=True)
    exe = nvcc()
    extra = list(extra or [])

    def compile_unit(item):
        name, flags = item
        obj = out_dir / (Path(name).stem + ".o")
        cmd = [exe, *ARCH, *COMMON, *flags, *extra, "-c", str(CSRC / name), "-o", str(obj)]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed for {name}:\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
        if verbose and (proc.stdout or proc.stderr):
            print(proc.stdout, proc.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=len(UNITS)) as pool:
        objs = list(pool.map(compile_unit, UNITS.items()))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [exe, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    import sys

    print(build_library(force="--force" in sys.argv, verbose=True,
                        extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None))
