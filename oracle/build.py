"""Build the FP64 C oracle (test infrastructure): oracle/libcpu_fdtd.so.

    python -m oracle.build

Compiled with OpenMP when the compiler supports it (single-threaded
otherwise; oracle_num_threads() reports which).
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu_fdtd.c"
OUT = HERE / "libcpu_fdtd.so"


def _compilers():
    seen = []
    for c in ("/usr/bin/gcc", os.environ.get("CC"), shutil.which("gcc"), "cc"):
        if c and c not in seen:
            seen.append(c)
    return seen


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    tmp = OUT.with_suffix(".so.tmp")
    last = None
    for omp in (["-fopenmp"], []):
        for cc in _compilers():
            cmd = [cc, "-O3", "-march=x86-64-v2", *omp, "-fPIC", "-shared", "-o", str(tmp), str(SRC)]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode == 0:
                os.replace(tmp, OUT)
                return OUT
            last = r.stderr
    raise RuntimeError(f"could not compile the C oracle: {last}")


if __name__ == "__main__":
    print(build(force=True))
