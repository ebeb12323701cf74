"""Build the sm_100a DG-MHD library in-tree: ``pp-es-dg-mhd_b200/libmhd_gpu.so``.

    nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -shared -Xcompiler -fPIC ...

The library exports the C ABI declared in ``include/mhd_gpu.h`` and links only the CUDA runtime.
Run ``python pp-es-dg-mhd_b200/build.py [--force] [--verbose]``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmhd_gpu.so")
SOURCES = ["mhd_gpu.cu", "tables.cpp"]
DEPS = SOURCES + ["common.cuh", "residual.cuh", "post.cuh", "misc.cuh", "setup.cuh", "tables.h",
                  "batch_impl.cuh", "server_impl.cuh"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    paths = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", "mhd_gpu.h")]
    for tuned in ("residual2_tuned.h", "post_tuned.h"):  # written by autotune.py
        if os.path.exists(os.path.join(CSRC, tuned)):
            paths.append(os.path.join(CSRC, tuned))
    return any(os.path.getmtime(p) > t for p in paths)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    if not force and not _stale():
        return LIB
    objs = []
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(bdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, *(extra_flags or []), "-I", os.path.join(ROOT, "include"),
               "-x", "cu" if src.endswith(".cu") else "c++", "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp", *objs,
           "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    build(force="--force" in sys.argv or extra is not None, verbose="--verbose" in sys.argv,
          extra_flags=extra)
    print(LIB)
