"""Build the sm_100a shared library libsimp_gpu.so in-tree with nvcc.

Every source compiles to its own object in parallel (under _build/), then
one link.  Variants:
  default   simp_b200/libsimp_gpu.so
  checked   simp_b200/libsimp_gpu_checked.so: device index checks
            (SIMP_CHECK_BOUNDS: a failed check sets a flag and skips the
            access, never traps; the entry point then returns
            SIMP_ERR_BOUNDS) and NVTX ranges around the passes
NVTX ranges alone in the default library: SIMP_NVTX=1 in the environment.

Usage: python -m simp_b200.build [--force] [--verbose-ptxas] [--checked]
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libsimp_gpu.so")
LIB_CHECKED = os.path.join(HERE, "libsimp_gpu_checked.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

VARIANTS = {
    "default": (LIB, []),
    "checked": (LIB_CHECKED, ["-DSIMP_CHECK_BOUNDS", "-DSIMP_NVTX"]),
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list[str]:
    # the system g++ (a CXX from the environment may lack its runtime specs)
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                  glob.glob(os.path.join(INCLUDE, "*.h")))


def up_to_date(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


def _flags(variant: str) -> list[str]:
    extra = list(VARIANTS[variant][1])
    if variant == "default" and os.environ.get("SIMP_NVTX") == "1":
        extra.append("-DSIMP_NVTX")
    return [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
            "-fvisibility=hidden", "-I", INCLUDE, *host_compiler(), *extra]


def build(force: bool = False, ptxas_verbose: bool = False, variant: str = "default") -> str:
    lib = VARIANTS[variant][0]
    if not force and up_to_date(lib):
        return lib
    objdir = os.path.join(ROOT, "_build", variant)
    os.makedirs(objdir, exist_ok=True)
    flags = _flags(variant) + (["-Xptxas", "-v"] if ptxas_verbose else [])

    def compile_one(src: str) -> str:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        subprocess.run([nvcc(), *flags, "-c", src, "-o", obj], check=True)
        return obj

    srcs = sources()
    # the largest translation units first
    srcs.sort(key=lambda p: -os.path.getsize(p))
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_one, srcs))
    cmd = [nvcc(), *ARCH, "-shared", *host_compiler(), "-o", lib + ".tmp", *sorted(objs), "-lcudart", "-ldl"]
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    v = "checked" if "--checked" in sys.argv else "default"
    build(force="--force" in sys.argv, ptxas_verbose="--verbose-ptxas" in sys.argv, variant=v)
    print(VARIANTS[v][0])
