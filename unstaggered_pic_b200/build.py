"""Build recipe for libupic.so, the sm_100a CUDA library behind include/upic.h.

    python -m unstaggered_pic_b200.build          # builds unstaggered_pic_b200/libupic.so and upic_run

nvcc compiles every source for sm_100a (it cross-compiles without a GPU);
the library links the CUDA runtime statically, so it loads next to any
PyTorch build.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libupic.so")
RUN = os.path.join(HERE, "upic_run")
BUILD = os.path.join(ROOT, "_build")

SOURCES = ["fft.cu", "sort.cu", "explicit.cu", "mixed.cu", "implicit.cu", "guess_net.cu", "api.cu", "api_implicit.cu",
           "ensemble.cu", "noalloc.cu", "generate.cpp", "p3_init.cpp"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "--expt-relaxed-constexpr",
]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose=False, ptxas_info=False):
    """Compile each source to an object under _build/ and link libupic.so."""
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "upic.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not ptxas_info and _newer(obj, [path] + headers):
            continue
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", path, "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if not _newer(OUT, objs) or ptxas_info:
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    # upic_run: the deck-driven driver (host C++ over the C ABI)
    srcs = [os.path.join(CSRC, "upic_run.cpp"), os.path.join(CSRC, "run_nonrel.cpp"),
            os.path.join(CSRC, "run_p3.cpp")]
    if not _newer(RUN, srcs + [OUT, os.path.join(ROOT, "include", "upic.h")]):
        cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include")] + srcs + ["-o", RUN,
               "-L", HERE, "-lupic", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
