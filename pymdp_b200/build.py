"""Build ``libpymdp_b200.so`` (sm_100a) in-tree with nvcc.

    python -m pymdp_b200.build          # or: python pymdp_b200/build.py

The library is a plain C-ABI shared object (``include/pymdp_b200.h``); the
CUDA runtime is linked statically (nvcc's default), so loading it needs no
GPU and no libcudart on the library path. Rebuilds when any source is newer than the .so.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpymdp_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(args):
    cmd, src = args
    res = subprocess.run(cmd, capture_output=True, text=True)
    return src, res.returncode, res.stdout + res.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile each source to an object in ``_build/`` (in parallel; only the
    stale ones), then link the shared library."""
    from concurrent.futures import ThreadPoolExecutor

    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "pymdp_b200.h")]
    deps = sources() + headers
    if not force and not _stale(LIB, deps):
        return LIB
    obj_dir = os.path.join(ROOT, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
             "-Xptxas", "-v" if verbose else "-O3"]
    jobs, objs = [], []
    for src in sources():
        obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append(([nvcc_path(), *flags, "-c", "-o", obj, src], src))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for src, rc, log in ex.map(_compile, jobs):
            if rc != 0:
                raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n" + log)
            if verbose:
                sys.stderr.write(f"== {os.path.basename(src)}\n" + log)
    res = subprocess.run([nvcc_path(), *ARCH, "--shared", "-o", LIB + ".tmp", *objs], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
