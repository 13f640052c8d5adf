"""Build the sm_100a shared library of the package in-tree.

    python -m pulsesuite_b200.build        # -> pulsesuite_b200/libpulsesuite_b200.so

nvcc cross-compiles for sm_100a without a GPU.  The library has a plain C
ABI (include/pulsesuite_b200.h) and links only the CUDA runtime.
"""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpulsesuite_b200.so")
SOURCES = ["capi.cu", "coulomb.cu", "sbe_f64.cu", "sbe_full.cu", "sbe_split.cu",
           "sbe_split_wire.cu", "wirespace_host.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps.append(os.path.join(REPO, "include", "pulsesuite_b200.h"))
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    # host code without fused multiply-adds (wirespace_host.cu reproduces
    # numpy's complex arithmetic operation by operation)
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler",
           "-fPIC,-ffp-contract=off",
           "-I", os.path.join(REPO, "include"), "-o", LIB + ".tmp", *sources(), "-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
