"""Build libbsofi_b200.so (FP64) and libbsofi_b200_fp32.so (the reference's
single-precision API over the same device pipeline) in-tree: sm_100a CUDA
kernels + the host C layer.

    python -m bsofi_b200.build          # or bsofi_b200.build.build()

nvcc compiles every kernel file for sm_100a (-gencode arch=compute_100a,
code=sm_100a), gcc compiles the host C layer, nvcc links each shared library
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

CU_SOURCES = ["kernels_bsof.cu", "kernels_bsoi.cu", "kernels_bstri.cu", "kernels_panel.cu", "kernels_tri.cu", "kernels_gemm.cu", "pipeline.cu", "kernels_dqmc.cu", "autotune.cu", "noalloc.cu", "kernels_ozaki.cu"]
C_SOURCES = ["bsofi_api.c", "batch.c", "server.c"]
# The single-precision library: the same device objects, the float API and
# its conversion kernels.
LIB32 = os.path.join(HERE, "libbsofi_b200_fp32.so")
CU_SOURCES_32 = ["kernels_convert.cu"]
C_SOURCES_32 = ["bsofi_api_fp32.c"]
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
    headers.append(os.path.join(ROOT, "include", "bsofi_b200_fp32.h"))

    def cu_obj(src):
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + headers):
            cmd = [nvcc] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                                   "-Xcompiler", "-fvisibility=hidden", "-I", CSRC, "-c", s, "-o", o]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            _run(cmd, verbose)
        return o

    def c_obj(src):
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + headers):
            _run(["gcc", "-O2", "-std=c99", "-D_GNU_SOURCE", "-fPIC", "-Wall", "-Wno-unused-function",
                  "-I", os.path.join(cuda, "include"), "-I", CSRC, "-c", s, "-o", o], verbose)
        return o

    dev = [cu_obj(src) for src in CU_SOURCES]
    objs = dev + [c_obj(src) for src in C_SOURCES]
    if force or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"], verbose)
    objs32 = dev + [cu_obj(src) for src in CU_SOURCES_32] + [c_obj(src) for src in C_SOURCES_32]
    if force or _stale(LIB32, objs32):
        # Export exactly the names bsofi_b200_fp32.h declares.
        vs = os.path.join(BUILD, "fp32.map")
        with open(vs, "w") as f:
            f.write("{ global: %s; local: *; };\n" % "; ".join(fp32_exports()))
        _run([nvcc] + ARCH + ["-shared", "-o", LIB32] + objs32 +
             ["-Xlinker", "--version-script=" + vs, "-lpthread", "-ldl", "-lrt"], verbose)
    return LIB


def fp32_exports():
    """Function names declared in include/bsofi_b200_fp32.h."""
    import re
    with open(os.path.join(ROOT, "include", "bsofi_b200_fp32.h")) as f:
        text = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void|double|long long)\s+\**(\w+)\s*\(", text,
                                 flags=re.M)))


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv)
