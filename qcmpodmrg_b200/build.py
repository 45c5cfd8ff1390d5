"""Build the native libraries in-tree (sm_100a only).

  lib/libqcgpu.so  nvcc -gencode arch=compute_100a,code=sm_100a: kernels + host block maps
  lib/libqsym.so   g++: drop-in for the reference's ctypes/qsym.c symAllowed
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_SOURCES = ["bgemm.cu", "bgemm_tc.cu", "tcpanel.cu", "fiber.cu", "fgemm.cu", "pgemm.cu", "sigma_noalloc.cu", "mlp.cu",
                "blockmap.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(verbose_ptxas=False):
    os.makedirs(LIB, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    cmd = [NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                           "-I", CSRC, "-o", os.path.join(LIB, "libqcgpu.so")] + srcs
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    _run(cmd)
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC, "-o", os.path.join(LIB, "libqsym.so"),
          os.path.join(CSRC, "qsym_dropin.cpp"), os.path.join(CSRC, "blockmap.cpp")])


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
