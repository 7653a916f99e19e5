"""Builds libchili_b200.so (CUDA kernels + C ABI) in-tree for sm_100a.

    python -m chili_b200.build

nvcc cross-compiles without a GPU.  The library links the CUDA runtime
statically, so it does not depend on the runtime that torch ships.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libchili_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Translation units whose FP64 phase-space arithmetic must round as the
# reference's x86-64 build does: no multiply-add contraction (cancellations in
# invariant masses, boosts and two-body momenta near threshold amplify the
# different rounding of a fused multiply-add to ~1e-9). The tensor-core flow
# layers and the channel-weight network keep contraction.
NO_CONTRACT = {"chili_gpu.cu", "batch.cu", "flow.cu"}
SOURCES = ["chili_gpu.cu", "flow.cu", "flow_layers.cu", "flow_wide.cu", "flow_alpha.cu", "channel_program.cpp", "checkpoint.cu", "batch.cu", "construct.cpp"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_build(out=OUT):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "chili_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compiles every source to an object in parallel (chili_b200/_build/),
    then links the shared library."""
    if not force and not needs_build():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

    def compile_one(src):
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        extra = ["--fmad=false"] if src in NO_CONTRACT else []
        cmd = common + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    link = [nvcc(), *ARCH, "-shared", "-o", OUT + ".tmp", *objs]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
