"""Build the CUDA library in-tree for sm_100a (python -m grace_b200.build).

One translation unit (csrc/api.cu) with the kernels in headers; the shared
object is written next to this file so that it ships with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def build(verbose=False):
    out = os.path.join(HERE, "libgrace_b200.so")
    srcs = [os.path.join(HERE, "csrc", "api.cu")]
    deps = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
    deps.append(os.path.join(ROOT, "include", "grace_b200.h"))
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), *srcs, "-o", out]
    if verbose:
        cmd.append("-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
