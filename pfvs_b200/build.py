"""
Build of libpfvs_gpu.so for sm_100a, in tree (pfvs_b200/fp_kernel/), with
nvcc.  No fast-math: the search's rigorous error bounds assume IEEE
division and square root (FMA contraction only reduces rounding error).
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = [os.path.join(HERE, "csrc", "pfg_abi.cu"), os.path.join(HERE, "csrc", "pfg_static.cu")]
OUT = os.path.join(HERE, "fp_kernel", "libpfvs_gpu.so")
DEPS = [os.path.join(HERE, "csrc", f) for f in
        ("pfg_abi.cu", "pfg_static.cu", "pfg_int.cuh", "pfg_types.cuh", "pfg_setup.cuh",
         "pfg_search.cuh", "pfg_out.cuh", "pfg_pfv.cuh", "pfg_mu0.cuh", "pfg_zpk.cuh")] + [os.path.join(HERE, "..", "include", "pfvs_gpu.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-shared", "-Xcompiler", "-fPIC"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(force=False, verbose=False, extra=()):
    """Compile the library if any source is newer than it (or force)."""
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d)):
            return OUT
    cmd = [nvcc(), *NVCC_FLAGS, *extra, *SRCS, "-o", OUT]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
