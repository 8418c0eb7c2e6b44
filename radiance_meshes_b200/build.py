"""Builds librm_b200.so (the C-ABI rasterizer library) for sm_100a with nvcc.

The library is built in-tree (``radiance_meshes_b200/lib/``) so that it travels
with the source tree; nothing is JIT-compiled at import time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIBNAME = "librm_b200.so"
SOURCES = ["rm_capi.cu", "rm_project.cu", "rm_scan.cu", "rm_sort.cu", "rm_blend.cu", "rm_fine.cu", "rm_features.cu", "rm_tets.cu"]
HEADERS = ["rm_internal.cuh", os.path.join("..", "..", "include", "rm_capi.h")]

# --fmad=false: every fused multiply-add in the kernels is written explicitly
# (fmaf), which keeps the integer outputs reproducible (see rm_internal.cuh).
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo", "--fmad=false",
    "-Xcompiler", "-fPIC,-O2,-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def lib_path() -> str:
    return os.path.join(LIBDIR, LIBNAME)


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS]
    out = lib_path()
    if not force and not _stale(out, deps):
        return out
    def compile_one(src):
        obj = os.path.join(LIBDIR, os.path.basename(src).replace(".cu", ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, *(extra_flags or []), "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, cmd, r

    # the translation units are independent: compile them concurrently
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, srcs))
    objs = []
    for src, obj, cmd, r in results:
        if verbose:
            print(" ".join(cmd), flush=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, flush=True)
        objs.append(obj)
    tmp = out + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
           "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, out)
    for o in objs:
        os.remove(o)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
