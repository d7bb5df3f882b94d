"""Builds the CUDA library in-tree: reactphysics3d_b200/_lib/librp3dg.so.

sm_100a only.  Floating-point flags are part of the contract with the
reference engine's float build: no FMA contraction (--fmad=false), IEEE
division and square root, no flush-to-zero, and no contraction in host code
either (-ffp-contract=off) so the host-side mesh set-up matches too.

Every source is compiled to its own object in parallel (no relocatable
device code: each file's kernels are self-contained), then one link makes
the shared library.  narrowphase_events.cu is the event-counting build of
the narrow-phase kernels (measurement only).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "librp3dg.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["rp3dg_host.cu", "narrowphase.cu", "narrowphase_events.cu", "peak.cu", "axis_mlp.cu", "contacts.cu", "dynamics.cu",
           "broadphase.cu", "world.cu", "heightfield.cu", "raycast.cu", "debug.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FP_FLAGS = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-fopenmp", "-Xptxas", "-v"] + FP_FLAGS


def _compile(src, obj, defines):
    cmd = [NVCC] + FLAGS + [f"-D{d}" for d in defines] + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r


def build(verbose=False, out=LIB, defines=(), jobs=None):
    os.makedirs(os.path.dirname(out), exist_ok=True)
    tag = "_".join(d.replace("=", "-") for d in defines) or "default"
    objdir = os.path.join(OBJDIR, tag)
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, s.replace(".cu", ".o")) for s in SOURCES]
    with ThreadPoolExecutor(max_workers=jobs or min(len(SOURCES), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda so: _compile(so[0], so[1], defines), zip(SOURCES, objs)))
    log = []
    for src, r in results:
        log.append(r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "--shared", "-Xcompiler", "-fPIC,-fopenmp"] + objs + \
           ["-o", out, "-lcudart", "-lgomp"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking librp3dg.so")
    if verbose:
        sys.stdout.write("".join(log))
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
