"""Builds the in-tree CUDA library for sm_100a (and the oracle for the tests).

    python -m gascoignelib_b200.build
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
# translation units: level set-up, the cycle, the GMRES drivers, the C-ABI
SRC = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]
DEPS = SRC + [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
              if f.endswith(".cuh")] + [os.path.join(ROOT, "include", "gascoigne_b200.h")]
OUT = os.path.join(HERE, "_lib", "libgascoigne_b200.so")
OBJ = os.path.join(HERE, "_lib", "obj")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
              "-std=c++17", "-Xcompiler", "-fPIC", "-Xfatbin", "-compress-all"]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build_library(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t for d in DEPS):
            return OUT
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    objs, procs = [], []
    for src in SRC:  # the units compile in parallel
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc] + NVCC_FLAGS + ["-c", "-o", obj, src]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                            text=True)))
        objs.append(obj)
    errors = []
    for cmd, p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            errors.append(" ".join(cmd) + "\n" + out + err)
        elif verbose:
            print(" ".join(cmd))
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    if verbose:
        print(" ".join(cmd))
    return OUT


def build_oracle() -> None:
    """Compiles the oracle's C restatement and, when the reference sources are
    present, the reference CPU solver (test infrastructure only)."""
    cmd = ["make", "-C", os.path.join(ROOT, "oracle")]
    ref = os.environ.get("GB_REFERENCE_SRC", "/root/reference/src")
    if os.path.isdir(ref):
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True, capture_output=True)


def build(force: bool = False) -> None:
    build_library(force=force)
    build_oracle()


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(OUT)
