"""Builds the CUDA library in-tree: reactphysics3d_b200/_lib/librp3dg.so.

sm_100a only.  Floating-point flags are part of the contract with the
reference engine's float build: no FMA contraction (--fmad=false), IEEE
division and square root, no flush-to-zero, and no contraction in host code
either (-ffp-contract=off) so the host-side mesh set-up matches too.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "librp3dg.so")
SOURCES = ["rp3dg_host.cu", "narrowphase.cu", "axis_mlp.cu", "contacts.cu", "dynamics.cu", "broadphase.cu", "world.cu", "heightfield.cu", "raycast.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FP_FLAGS = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-fopenmp", "--shared", "-Xptxas", "-v"] + FP_FLAGS


def build(verbose=False, out=LIB, defines=()):
    os.makedirs(os.path.dirname(out), exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    cmd = [NVCC] + FLAGS + [f"-D{d}" for d in defines] + srcs + ["-o", out, "-lcudart", "-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building librp3dg.so")
    if verbose:
        sys.stdout.write(r.stderr)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
