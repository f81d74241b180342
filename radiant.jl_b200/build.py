"""Builds libradiant_b200.so (the CUDA library) in-tree for sm_100a.

    python radiant.jl_b200/build.py [--force] [--verbose]

nvcc compiles every csrc/*.cu (the host ABI in rb_capi.cu and each persistent kernel in its own
rb_kernel_*.cu) to an object in parallel, then links one shared library with a C ABI; the
output lands in radiant_b200/lib/ so it travels with the source tree.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "radiant_b200", "lib", "libradiant_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh", ".h"))] + [
        os.path.join(HERE, "..", "include", "radiant_b200.h")]


def build(force: bool = False, verbose: bool = False) -> str:
    if (not force and os.path.exists(OUT)
            and os.path.getmtime(OUT) >= max(os.path.getmtime(s) for s in sources())):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
             "--expt-relaxed-constexpr", "--extended-lambda", "-diag-suppress=128"]
    if verbose:
        flags.append("-Xptxas=-v")
    units = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    objs = [os.path.join(objdir, u[:-3] + ".o") for u in units]

    def compile_one(k):
        subprocess.check_call([NVCC, *flags, "-c", os.path.join(CSRC, units[k]), "-o", objs[k]])

    with ThreadPoolExecutor(max_workers=len(units)) as ex:
        list(ex.map(compile_one, range(len(units))))
    subprocess.check_call([NVCC, *ARCH, "-shared", *objs, "-o", OUT, "-lcudart"])
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
