"""Build libptstokes.so (sm_100a) in-tree with nvcc.

    python pseudotransientstokes.jl_b200/build.py [--force] [--verbose-ptxas]

FP64 kernels are compiled with --fmad=false (no multiply-add contraction) so they round
exactly like the reference's Float64 arithmetic; FP32 kernels keep FMA contraction.
The shared library links the CUDA runtime statically and exports only the C ABI of
include/ptstokes.h.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libptstokes.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]

# translation unit -> extra flags
UNITS = {
    "pts_kernels64.cu": ["--fmad=false"],
    "pts_noalloc.cu": ["--fmad=false"],
    "pts_zstage.cu": ["--fmad=false"],
    "pts_kernels32.cu": [],
    "pts_abi.cu": [],
    "pts_batch.cu": [],
}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, ptxas_verbose=False, quiet=False, defines=(), out=None):
    """Compile and link libptstokes.so. `defines` (NAME=VALUE) and `out` build a variant
    library elsewhere (for A/B timing of compile-time tunables); the default is in-tree."""
    global BUILD, LIB
    if out:
        BUILD = os.path.join(os.path.dirname(os.path.abspath(out)), "_build_variant")
        LIB = os.path.abspath(out)
        force = True
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    dflags = [f"-D{d}" for d in defines]
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "ptstokes.h"))
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src, *headers, __file__]):
            cmd = [nvcc(), *ARCH, *COMMON, *dflags, *extra, "-c", src, "-o", obj]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            if not quiet:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"]
        if not quiet:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--define", action="append", default=[], help="NAME=VALUE passed as -D to nvcc")
    ap.add_argument("--out", default=None, help="write the library here instead of in-tree")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.verbose_ptxas, defines=a.define, out=a.out))
    sys.exit(0)
