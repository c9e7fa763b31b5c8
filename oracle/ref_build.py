"""Build recipe for ``oracle/_ref``: the reference's own CPU FFI kernels,
compiled unchanged from their sources, as a CPU timing baseline and second
cross-check (test infrastructure; nothing in the product path loads it).

    python -m oracle.ref_build          # needs the reference sources at REF_SRC

Sources (from the reference tree, not copied): ``pymdp/ffi/neg_efe/
neg_efe_cpu_entry.cc`` and ``neg_efe_cpu_pipeline.cc`` (NegEfeCpu) and
``pymdp/ffi/fpi/fpi_cpu_runner.cc`` (FpiCpu), with the headers they include,
plus ``oracle/refbuild/ref_cpu_shim.cc`` (C entry points). The reference's
build gets ``xla/ffi/api/ffi.h`` from jaxlib (``CMakeLists.txt:42-56``);
jaxlib is absent here, so ``oracle/refbuild/include`` supplies a
project-written stand-in for the five types the CPU sources use.

Flags follow the reference's release build (``CMakeLists.txt``: ``-O3
-ffast-math``, ``-march=native``, LTO, OpenMP), except that ``-march`` is
fixed so the library runs on another host: ``x86-64-v3`` (AVX2 + FMA, the
reference's default SIMD path) and ``x86-64-v4`` (AVX-512 for the compiler;
the reference's own AVX-512 intrinsics stay off, as in its default build).
``load()`` picks v4 when the host CPU has AVX-512F, which is what
``-march=native`` would have given on that host.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REF_SRC = os.environ.get("PYMDP_REF_FFI", "/root/reference/pymdp/ffi")
SOURCES = ["neg_efe/neg_efe_cpu_entry.cc", "neg_efe/neg_efe_cpu_pipeline.cc", "fpi/fpi_cpu_runner.cc"]
VARIANTS = {"v3": "x86-64-v3", "v4": "x86-64-v4"}


def lib_path(variant: str) -> str:
    return os.path.join(OUT, f"libpymdp_ref_cpu_{variant}.so")


def build(force: bool = False) -> bool:
    """Compile both variants when the reference sources are present; returns
    whether the libraries exist afterwards."""
    if not os.path.isdir(REF_SRC):
        return all(os.path.exists(lib_path(v)) for v in VARIANTS)
    os.makedirs(OUT, exist_ok=True)
    srcs = [os.path.join(REF_SRC, s) for s in SOURCES] + [os.path.join(HERE, "refbuild", "ref_cpu_shim.cc")]
    deps = srcs + [os.path.join(HERE, "refbuild", "include", "xla", "ffi", "api", "ffi.h")]
    procs = []
    for v, march in VARIANTS.items():
        lib = lib_path(v)
        if not force and os.path.exists(lib) and all(os.path.getmtime(d) <= os.path.getmtime(lib) for d in deps):
            continue
        cmd = ["g++", "-std=c++17", "-O3", "-ffast-math", f"-march={march}", "-fopenmp", "-flto", "-fPIC", "-shared",
               "-w", "-I", os.path.join(HERE, "refbuild", "include"), "-I", REF_SRC, "-o", lib + ".tmp", *srcs]
        procs.append((lib, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for lib, pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError(f"reference CPU build failed:\n{out}")
        os.replace(lib + ".tmp", lib)
    return True


def host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " avx512f " in line + " "
    except OSError:
        pass
    return False


def variant() -> str:
    return "v4" if host_has_avx512() and os.path.exists(lib_path("v4")) else "v3"


_LIB = None


def load():
    """The reference CPU library for this host (raises when it was not built)."""
    global _LIB
    if _LIB is None:
        path = lib_path(variant())
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run python -m oracle.ref_build where the reference is present")
        lib = ctypes.CDLL(path)
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_neg_efe_cpu.restype = ctypes.c_int
        lib.ref_fpi_cpu.restype = ctypes.c_int
        _LIB = lib
    return _LIB


if __name__ == "__main__":
    ok = build(force="--force" in sys.argv)
    print("built" if ok else "reference sources absent and no prebuilt library", lib_path("v3"), lib_path("v4"))
