"""Builds the sm_100a shared library libproteus_gpu.so in-tree with nvcc.

Every .cu file under csrc/ is compiled separately (so that a change rebuilds one
object) and linked with the CUDA runtime into proteusgpu_b200/libproteus_gpu.so.
FP64 files are compiled with -fmad=false: the parity contract with the
reference's CPU build requires unfused multiply/add sequences.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libproteus_gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# per-file extra flags; files not listed get the FP64 parity flags
FAST_MATH_FILES: set[str] = {"diag.cu"}


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def sources() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _flags(src: str, verbose_ptxas: bool) -> list[str]:
    f = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-I", CSRC,
         "-I", os.path.join(HERE, "..", "include")] + ARCH
    f += ["-fmad=true"] if src in FAST_MATH_FILES else ["-fmad=false"]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def build(force: bool = False, verbose_ptxas: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "proteus_gpu.h"))
    hdr_time = max(os.path.getmtime(h) for h in headers)
    procs, objs = [], []
    for src in sources():
        spath = os.path.join(CSRC, src)
        opath = os.path.join(OBJ, src[:-3] + ".o")
        objs.append(opath)
        if (not force and os.path.exists(opath)
                and os.path.getmtime(opath) >= max(os.path.getmtime(spath), hdr_time)):
            continue
        cmd = [nvcc(), "-c", spath, "-o", opath] + _flags(src, verbose_ptxas)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if jobs and len(procs) >= jobs:
            _wait(procs, verbose_ptxas)
            procs = []
    _wait(procs, verbose_ptxas)
    if (force or not os.path.exists(LIB)
            or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


def _wait(procs, verbose):
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, text))
        elif verbose and text.strip():
            print(f"--- {src}\n{text}")
    if failed:
        msg = "\n".join(f"--- {s}\n{t}" for s, t in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
    print(LIB)
