"""Build libcdns_cuda.so in-tree for sm_100a (nvcc, no JIT).

Usage: python channel-dns_b200/build.py [--debug]
The library lands beside the Python package: channel-dns_b200/cdns/libcdns_cuda.so
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "cdns", "libcdns_cuda.so")
SOURCES = ["context.cu", "chebyshev.cu", "transforms.cu", "solver.cu", "solver_setup.cu", "layout.cu", "noalloc.cu",
           "adjoint.cu", "adjoint_run.cu", "output.cu", "tune.cu",
           "field_files.cu", "pencil.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


# Per-file nvcc flags.  The solver setup keeps the reference's rounding of each
# operation (no FMA contraction): it feeds differences that cancel to 1e-6 of
# their terms.  The step solve contracts (its results stay within 2e-13 of the
# reference's after 1000 Re_tau180 steps).
FILE_FLAGS = {"solver_setup.cu": ["-fmad=false"]}


def build(verbose: bool = False, extra=None) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps.append(os.path.join(ROOT, "include", "cdns.h"))
    deps.append(os.path.abspath(__file__))
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps) \
            and not extra:
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in SOURCES:
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", os.path.join(ROOT, "include"), *FILE_FLAGS.get(s, []), *(extra or []),
               "-c", os.path.join(CSRC, s), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    # the CUDA runtime is linked statically: the library always runs on the
    # runtime it was compiled against, whatever libcudart the host process loads
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", OUT, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    print(build(verbose=True, extra=extra))
