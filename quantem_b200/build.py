"""Build libptycho_b200.so in-tree with nvcc for sm_100a.

    python -m quantem_b200.build [--force]

Each translation unit under ``csrc/`` is compiled in parallel to an object file
under ``csrc/_build/`` and linked into ``lib/libptycho_b200.so``.  A build stamp
(hash of sources, headers and flags) skips the rebuild when nothing changed.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(CSRC, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libptycho_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libptycho_b200")


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_hash() -> bytes:
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for f in sorted(os.listdir(d)):
            if f.endswith((".cuh", ".h")):
                with open(os.path.join(d, f), "rb") as fh:
                    h.update(f.encode() + fh.read())
    h.update(" ".join(ARCH + NVCC_FLAGS).encode())
    return h.digest()


def _obj_stamp(src: str) -> str:
    h = hashlib.sha256(_headers_hash())
    with open(os.path.join(CSRC, src), "rb") as fh:
        h.update(fh.read())
    return h.hexdigest()


def _stamp() -> str:
    h = hashlib.sha256(_headers_hash())
    for src in _sources():
        h.update(_obj_stamp(src).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every CUDA translation unit and link the shared library."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    stamp_file = os.path.join(BUILD, "stamp")
    stamp = _stamp()
    if not force and os.path.exists(LIB) and os.path.exists(stamp_file):
        with open(stamp_file) as fh:
            if fh.read().strip() == stamp:
                return LIB
    nvcc = _nvcc()
    extra = ["-Xptxas", "-v"] if ptxas_info else []

    def compile_one(src):
        obj = os.path.join(BUILD, src[:-3] + ".o")
        ostamp = obj + ".stamp"
        want = _obj_stamp(src)
        if not force and not ptxas_info and os.path.exists(obj) and os.path.exists(ostamp):
            with open(ostamp) as fh:
                if fh.read().strip() == want:
                    return src, obj, subprocess.CompletedProcess([], 0, "", "")
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            with open(ostamp, "w") as fh:
                fh.write(want)
        return src, obj, r

    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, _sources()))
    objs = []
    for src, obj, r in results:
        if verbose or ptxas_info:
            sys.stdout.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        objs.append(obj)
    cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    with open(stamp_file, "w") as fh:
        fh.write(stamp)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose=True, ptxas_info="--ptxas" in sys.argv))
