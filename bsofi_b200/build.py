"""Build libbsofi_b200.so in-tree: sm_100a CUDA kernels + the host C layer.

    python -m bsofi_b200.build          # or bsofi_b200.build.build()

nvcc compiles every kernel file for sm_100a (-gencode arch=compute_100a,
code=sm_100a), gcc compiles the host C layer, nvcc links one shared library
with the CUDA runtime linked statically.  Objects go to bsofi_b200/_build/.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbsofi_b200.so")
ROOT = os.path.dirname(HERE)

CU_SOURCES = ["kernels_bsof.cu", "kernels_bsoi.cu", "kernels_bstri.cu", "kernels_panel.cu", "kernels_tri.cu", "kernels_gemm.cu", "pipeline.cu", "kernels_dqmc.cu", "autotune.cu", "noalloc.cu"]
C_SOURCES = ["bsofi_api.c", "batch.c", "server.c"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cuda_home():
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False, ptxas_verbose=False):
    cuda = _cuda_home()
    nvcc = os.path.join(cuda, "bin", "nvcc")
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "bsofi_b200.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                                   "-Xcompiler", "-fvisibility=hidden", "-I", CSRC, "-c", s, "-o", o]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            _run(cmd, verbose)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            _run(["gcc", "-O2", "-std=c99", "-D_GNU_SOURCE", "-fPIC", "-Wall", "-Wno-unused-function",
                  "-I", os.path.join(cuda, "include"), "-I", CSRC, "-c", s, "-o", o], verbose)
    if force or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv)
