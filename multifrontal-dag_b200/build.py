"""Build libmfdag.so (sm_100a) in-tree with nvcc.

    python multifrontal-dag_b200/build.py [--debug]

Sources: csrc/analysis.cpp (host symbolic analysis), csrc/ordering.cpp (nested
dissection ordering), csrc/partition.cpp (subtree-to-GPU mapping),
csrc/kernels.cu (device
kernels), csrc/update_tc.cu (FP32 tcgen05 update), csrc/api.cu (C ABI, plan,
launch sequences), csrc/noalloc.cu (allocation-free fronts), csrc/input.cu
(Matrix Market, COO -> CCS on the GPU, CSR input).  Output:
multifrontal-dag_b200/mfdag/libmfdag.so, loaded by mfdag/hppllt.py.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "mfdag", "libmfdag.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["analysis.cpp", "ordering.cpp", "partition.cpp", "kernels.cu", "update_tc.cu", "api.cu", "noalloc.cu",
           "input.cu"]


def build(debug: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    if os.path.exists(OUT) and not debug:
        newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(CSRC, h) for h in os.listdir(CSRC)]
                     + [os.path.join(os.path.dirname(HERE), "include", "mfdag.h")])
        if os.path.getmtime(OUT) >= newest:
            return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    opt = ["-O0", "-g", "-G"] if debug else ["-O3"]
    common = ["-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", CSRC,
              "-I", os.path.join(os.path.dirname(HERE), "include")] + opt
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [NVCC, "-c", s, "-o", o] + common + ARCH
        if s.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        else:
            cmd = ["g++", "-x", "c++", "-c", s, "-o", o, "-std=c++17", "-O3", "-fPIC", "-fvisibility=hidden", "-I", CSRC,
                   "-I", os.path.join(os.path.dirname(HERE), "include")]
        subprocess.run(cmd, check=True)
        objs.append(o)
    link = [NVCC, "-shared", "-o", OUT] + objs + ARCH + ["-Xcompiler", "-fPIC"]
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    print(build(debug="--debug" in sys.argv, verbose="-v" in sys.argv))
