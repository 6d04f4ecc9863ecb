"""Build the CPU oracle (test infrastructure only): oracle/build/liboracle.so.

Tries the available C compilers with OpenMP first and falls back to a
single-threaded build when no OpenMP runtime links.  Also (re)builds the
reference CUDA extension into oracle/_ref/ when the reference sources are
present (oracle/build_ref.sh).

    python oracle/build.py [--ref]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle.c")
OUT = os.path.join(HERE, "build", "liboracle.so")
FLAGS = ["-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-std=c11", "-shared"]


def _compilers():
    seen = []
    for c in (os.environ.get("CC"), "x86_64-linux-gnu-gcc-13", "gcc-13", "gcc", "cc"):
        if c and shutil.which(c) and c not in seen:
            seen.append(c)
    return seen


def build_oracle(force: bool = False) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(SRC),
                                                                           os.path.getmtime(__file__)):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    errors = []
    for omp in (["-fopenmp"], []):
        for cc in _compilers():
            tmp = OUT + ".tmp"
            r = subprocess.run([cc] + FLAGS + omp + ["-o", tmp, SRC, "-lm"], capture_output=True, text=True)
            if r.returncode == 0:
                os.replace(tmp, OUT)
                return OUT
            errors.append(f"{cc} {' '.join(omp)}: {r.stderr.strip()[-300:]}")
    raise RuntimeError("could not build the oracle:\n" + "\n".join(errors))


def build_reference() -> bool:
    """Build oracle/_ref/dose_kernels*.so from the reference sources if they
    are present; returns False when they are not."""
    script = os.path.join(HERE, "build_ref.sh")
    ref_root = os.environ.get("DOSECUDA_REFERENCE", "/root/reference")
    if not os.path.isdir(os.path.join(ref_root, "DoseCUDA", "dose_kernels")):
        return False
    ref_dir = os.path.join(HERE, "_ref")
    so = [f for f in os.listdir(ref_dir)] if os.path.isdir(ref_dir) else []
    if any(f.startswith("dose_kernels") and f.endswith(".so") for f in so):
        return True
    subprocess.run(["bash", script, ref_root], check=True, env=dict(os.environ, PYTHON=sys.executable))
    return True


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    if "--ref" in sys.argv:
        print("reference built:", build_reference())
