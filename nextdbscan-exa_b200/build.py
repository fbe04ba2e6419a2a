"""Builds libndb_b200.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ behind the C ABI of include/ndb_b200.h; no torch
extension machinery is involved, so the .so can be loaded by ctypes, cgo, JNI or a
C++ program alike.  Objects are compiled in parallel and cached by source mtime.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libndb_b200.so")
OBJDIR = os.path.join(HERE, "_build")

# Exactness: the reference's FP32 predicate has no FMA contraction and keeps
# denormals (g++ -O3 without -march/-ffast-math), so neither may the device code.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-ftz=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-I", INCLUDE, "-I", CSRC,
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime() -> float:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, obj: str, extra: list[str]) -> None:
    cmd = [nvcc_path(), *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compiles every .cu under csrc/ and links libndb_b200.so; returns its path."""
    extra = list(extra or [])
    os.makedirs(OBJDIR, exist_ok=True)
    hdr = _headers_mtime()
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        stale = force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr)
        if stale:
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            futs = [ex.submit(_compile, s, o, extra) for s, o in jobs]
            for f in futs:
                f.result()
    if jobs or not os.path.exists(LIB):
        cmd = [nvcc_path(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs,
               "-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB} ({len(jobs)} objects recompiled)")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
