"""Build the CPU oracle (test infrastructure only): oracle/build/liboracle.so.

Tries the available C compilers with OpenMP first and falls back to a
single-threaded build when no OpenMP runtime links.  Also (re)builds the
reference CUDA extension into oracle/_ref/ when the reference sources are
present (oracle/build_ref.sh).

    python oracle/build.py [--ref [REFERENCE_ROOT]]
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


def reference_root(explicit: str | None = None) -> str | None:
    """The reference checkout: the argument, else $DOSECUDA_REFERENCE, else a
    ``reference`` directory beside this repository; None when none of these
    holds the reference sources."""
    repo = os.path.dirname(HERE)
    for cand in (explicit, os.environ.get("DOSECUDA_REFERENCE"), os.path.join(os.path.dirname(repo), "reference")):
        if cand and os.path.isdir(os.path.join(cand, "DoseCUDA", "dose_kernels")):
            return cand
    return None


def build_reference(root: str | None = None) -> bool:
    """Build the reference checker into oracle/_ref/ (its CPython extension and
    the TERMA harness) from the reference sources if they are present;
    returns False when they are not."""
    script = os.path.join(HERE, "build_ref.sh")
    ref_root = reference_root(root)
    if ref_root is None:
        return False
    ref_dir = os.path.join(HERE, "_ref")
    have = set(os.listdir(ref_dir)) if os.path.isdir(ref_dir) else set()
    newest_src = max(os.path.getmtime(script), os.path.getmtime(os.path.join(HERE, "ref_terma.cu")))
    ok = (any(f.startswith("dose_kernels") and f.endswith(".so") for f in have) and "libref_terma.so" in have
          and os.path.getmtime(os.path.join(ref_dir, "libref_terma.so")) >= newest_src)
    if ok:
        return True
    subprocess.run(["bash", script, ref_root], check=True, env=dict(os.environ, PYTHON=sys.executable))
    return True


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    if "--ref" in sys.argv:
        i = sys.argv.index("--ref")
        print("reference built:", build_reference(sys.argv[i + 1] if len(sys.argv) > i + 1 else None))
