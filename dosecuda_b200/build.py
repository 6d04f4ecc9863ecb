"""Build recipe for the DoseCUDA B200 engine library (libdosecuda.so).

Compiles every ``csrc/*.cu`` translation unit for sm_100a with nvcc and links
them into ``dosecuda_b200/libdosecuda.so`` (in-tree, so the built library
travels with the source tree).  Objects are rebuilt only when a source or
header is newer than the library.

    python -m dosecuda_b200.build [--force] [--verbose]
    python -m dosecuda_b200.build --debug-bounds --out /tmp/libdosecuda_dbg.so

``--debug-bounds`` builds the bounds-checked variant (-DDC_DEBUG_BOUNDS: every
instrumented global access of the dose kernels checks its index and records
the first violation, read back by ``dc_debug_bounds``) into ``--out``, with its
objects beside it, leaving the in-tree library alone.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdosecuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
              "-I" + os.path.join(ROOT, "include")] + ARCH


def _nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdosecuda.so")
    return exe


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "dosecuda.h"))
    return hs


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths if os.path.exists(p)), default=0.0)


def build(force: bool = False, verbose: bool = False, extra_flags=None, out: str | None = None,
          debug_bounds: bool = False) -> str:
    """Compile and link libdosecuda.so (or ``out``); returns its path."""
    lib = os.path.abspath(out) if out else LIB
    obj_dir = (lib + "_obj") if out else OBJ
    srcs = _sources()
    hdr_time = _newest(_headers())
    if (not force and os.path.exists(lib)
            and os.path.getmtime(lib) >= max(_newest(srcs), hdr_time, os.path.getmtime(__file__))):
        return lib
    os.makedirs(obj_dir, exist_ok=True)
    nvcc = _nvcc()
    flags = NVCC_FLAGS + list(extra_flags or []) + (["-DDC_DEBUG_BOUNDS"] if debug_bounds else [])

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc] + flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, flush=True)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = lib + ".tmp"
    cmd = [nvcc, "-shared"] + ARCH + ["-Xcompiler", "-fPIC"] + objs + ["-o", tmp, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    ap.add_argument("--debug-bounds", action="store_true", help="bounds-checked variant (needs --out)")
    ap.add_argument("--out", default=None, help="library path (default: the in-tree libdosecuda.so)")
    a = ap.parse_args()
    if a.debug_bounds and not a.out:
        ap.error("--debug-bounds builds a separate library: give --out")
    path = build(force=a.force, verbose=a.verbose, extra_flags=["-Xptxas", "-v"] if a.ptxas_v else None,
                 out=a.out, debug_bounds=a.debug_bounds)
    print(path)
