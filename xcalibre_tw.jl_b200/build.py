"""Build libxcal.so in-tree (sm_100a) with nvcc.

    python xcalibre_tw.jl_b200/build.py [--verbose]

--fmad=false keeps every multiply and add separately rounded, the contract the
FP64 path's bitwise parity with the CPU oracle depends on (the kernels are
bandwidth bound, so fused multiply-adds would not make them faster).  The
persistent program (csrc/xcal_kernel.cu) is compiled once per instantiation
(components x scalar type), in parallel.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libxcal.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-Wno-deprecated-gpu-targets", "-O3", "-std=c++17", "--fmad=false", "-lineinfo",
         "-Xcompiler", "-fPIC,-O2,-ffp-contract=off", "--expt-relaxed-constexpr", "-diag-suppress=177"]
# instantiation tag -> (components, Krylov value type, resident CTAs per SM the
# register budget is sized for); the "o" builds trade spills for occupancy
INSTANCES = {"d1": (1, "double", 2), "d2": (2, "double", 2), "d3": (3, "double", 2), "f2": (2, "float", 2),
             "f3": (3, "float", 2), "d2o": (2, "double", 4), "d3o": (3, "double", 4), "f2o": (2, "float", 4),
             "f3o": (3, "float", 4)}
UNITS = [("xcal_kernel.cu", tag, ["-DXCAL_INST=" + tag, f"-DXCAL_NS={ns}", f"-DXCAL_T={t}", f"-DXCAL_MB={mb}"])
         for tag, (ns, t, mb) in INSTANCES.items()]
# the serving kernel of the 2D and 3D 4-CTA/SM builds, one unit each (compiled in parallel)
UNITS += [("xcal_kernel.cu", "s" + tag, ["-DXCAL_INST=" + tag, f"-DXCAL_NS={ns}", f"-DXCAL_T={t}",
                                         f"-DXCAL_MB={mb}", "-DXCAL_SERVE_ONLY"])
          for tag, (ns, t, mb) in INSTANCES.items() if mb == 4 and ns >= 2]
UNITS += [("xcal_launch.cu", None, []), ("xcal_ops.cu", None, []), ("xcal_operators.cu", None, []),
          ("xcal_api.cu", None, []),
          ("host_mesh.cpp", None, []), ("xcal_serve.cu", None, [])]


def build(verbose=False):
    import time
    t_start = time.time()   # sources are read from here on; objects are stamped with it
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "xcal.h"))
    newest_header = max(os.path.getmtime(h) for h in headers)
    procs, objs = [], []
    for src_name, tag, defs in UNITS:
        src = os.path.join(CSRC, src_name)
        obj = os.path.join(bdir, src_name + (f".{tag}" if tag else "") + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header):
            continue
        if src_name.endswith(".cpp"):
            cmd = [NVCC] + FLAGS + ["-x", "c++", "-c", src, "-o", obj]
        else:
            cmd = [NVCC] + ARCH + FLAGS + defs + ["-c", src, "-o", obj]
            if verbose:
                cmd += ["-Xptxas", "-v"]
        procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError("compile failed: " + " ".join(failed[0]))
    # an object is as new as the sources it was compiled from: a source edited
    # while the build ran is newer than its object and compiles again next time
    for cmd, p in procs:
        obj = cmd[cmd.index("-o") + 1]
        os.utime(obj, (t_start, t_start))
    subprocess.run([NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart", "-lpthread"], check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
