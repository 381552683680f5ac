"""Build recipe for ``oracle/_ref/librcabeam_ref.so`` -- TEST INFRASTRUCTURE ONLY.

Compiles the reference's own CUDA core, unchanged, from its sources where
they lie (``src/rcabeam/core.cu`` and ``src/rcabeam/ensemble.cu`` with
``include/rcabeam.h``, the two translation units of the reference's
``rcabeam_core`` library, CMakeLists.txt:17-19) into a shared library for
sm_100a.  The GPU tests load it through ctypes to pin the B200 kernels against
the reference kernels on the same device inputs and to time them side by side.

Nothing is copied into the repository: the output goes to ``oracle/_ref/``,
which git ignores.  When the reference sources are absent (on a machine that
only runs the prebuilt files) the recipe leaves an existing build untouched.

    python oracle/build_ref.py <reference_root>     (or RCABEAM_REFERENCE=<reference_root>)
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref" / "librcabeam_ref.so"
SOURCES = ("src/rcabeam/core.cu", "src/rcabeam/ensemble.cu")


def build(reference_root: Path, verbose: bool = False) -> Path | None:
    sources = [reference_root / s for s in SOURCES]
    header = reference_root / "include" / "rcabeam.h"
    if not header.exists() or not all(s.exists() for s in sources):
        return OUT if OUT.exists() else None
    if OUT.exists() and all(OUT.stat().st_mtime >= p.stat().st_mtime for p in (*sources, header)):
        return OUT
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix(".tmp.so")
    # -Bsymbolic keeps the reference's internal calls inside this library even
    # though the B200 library exports the same C names in the same process.
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-Xlinker", "-Bsymbolic", "-I", str(reference_root / "include"),
           *map(str, sources), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RCABEAM_REFERENCE")
    if not root:
        sys.exit("usage: build_ref.py <reference checkout> (or set RCABEAM_REFERENCE)")
    print(build(Path(root), verbose=True))
