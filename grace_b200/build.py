"""Build the CUDA library in-tree for sm_100a (python -m grace_b200.build).

One translation unit (csrc/api.cu) with the kernels in headers; the shared
objects are written next to this file so that they ship with the source
tree.  Two builds of the same sources:
  libgrace_b200.so        the product (nvcc's default contraction of
                          multiply-adds into FMAs)
  libgrace_b200_exact.so  every multiply and add rounded on its own
                          (-fmad=false), as the CPU oracle is compiled
                          (-ffp-contract=off): parity tests use it to tell a
                          rounding difference from a logic difference
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
VARIANTS = {"default": ("libgrace_b200.so", []),
            "exact": ("libgrace_b200_exact.so", ["-fmad=false"])}


def _command(variant, verbose=False):
    name, extra = VARIANTS[variant]
    out = os.path.join(HERE, name)
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", *extra, "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "csrc", "api.cu"), "-o", out]
    if verbose:
        cmd.append("-Xptxas=-v")
    return out, cmd


def _stale(out):
    deps = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
    deps.append(os.path.join(ROOT, "include", "grace_b200.h"))
    return not os.path.exists(out) or any(os.path.getmtime(out) < os.path.getmtime(d) for d in deps)


def build(verbose=False, variants=("default", "exact")):
    """Compile the stale variants (in parallel); returns their paths."""
    procs, outs = [], []
    for v in variants:
        out, cmd = _command(v, verbose)
        outs.append(out)
        if _stale(out):
            procs.append((cmd, subprocess.Popen(cmd)))
    for cmd, p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    return outs


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
