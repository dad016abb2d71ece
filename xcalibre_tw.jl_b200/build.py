"""Build libxcal.so in-tree (sm_100a) with nvcc.

    python xcalibre_tw.jl_b200/build.py [--verbose]

--fmad=false keeps every multiply and add separately rounded, the contract the
FP64 path's bitwise parity with the CPU oracle depends on (the kernels are
bandwidth bound, so fused multiply-adds would not make them faster).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libxcal.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-Wno-deprecated-gpu-targets", "-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
         "--expt-relaxed-constexpr"]
SOURCES = ["xcal_kernel.cu", "xcal_ops.cu", "xcal_api.cu", "host_mesh.cpp"]


def build(verbose=False):
    objs = []
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(bdir, s + ".o")
        deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
        deps.append(os.path.join(HERE, "..", "include", "xcal.h"))
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(d) for d in deps):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
            if verbose and s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if s.endswith(".cpp"):
                cmd = [NVCC] + FLAGS + ["-x", "c++", "-c", src, "-o", obj]
            subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
