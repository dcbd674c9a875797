"""Builds the CUDA engine library in-tree: optflow-soil_b200/lib/liboptflow_cuda.so (sm_100a).

    python optflow-soil_b200/build.py [--verbose]

Every kernel is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``); the CUDA runtime is
linked statically so the library needs only the driver on the machine that loads it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "liboptflow_cuda.so")
SOURCES = ["engine.cu", "fft.cu", "fine.cu", "poc.cu", "finish.cu", "synth.cu", "noalloc.cu", "gemm_sm100.cu", "net.cu",
           "net_api.cu", "proposal.cu", "warp_tma.cu", "tma.cu",
           "accumulate_tma.cu"]
# sources compiled against the CUTLASS / CuTe header tree (its sm100 GEMM collectives)
CUTLASS_SOURCES = {"gemm_sm100.cu"}
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-cudart", "static"]


def cutlass_include():
    """The CUTLASS / CuTe headers vendored with flashinfer (CUTLASS 4.x, sm100 collectives)."""
    import site
    roots = list(site.getsitepackages()) + [site.getusersitepackages()]
    for r in roots:
        d = os.path.join(r, "flashinfer", "data", "cutlass", "include")
        if os.path.exists(os.path.join(d, "cutlass", "gemm", "collective", "sm100_mma_warpspecialized.hpp")):
            return d
    raise RuntimeError("CUTLASS headers with the sm100 collectives not found (flashinfer/data/cutlass/include)")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    objdir = os.path.join(HERE, "lib", "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    inc_dir = os.path.join(os.path.dirname(HERE), "include")
    headers += [os.path.join(inc_dir, f) for f in os.listdir(inc_dir) if f.endswith(".h")]
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            inc = ["-I" + cutlass_include(), "-diag-suppress", "20012"] if s in CUTLASS_SOURCES else []
            cmd = [NVCC] + FLAGS + inc + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objs):
        subprocess.run([NVCC, "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-o", LIB] + objs, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
