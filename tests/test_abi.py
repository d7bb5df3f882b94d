"""The C-ABI library loads and exports every function include/rp3dg.h
declares; without a GPU it refuses to create a context (no CPU fallback)."""
import ctypes as C
import os
import subprocess

import pytest

from reactphysics3d_b200 import engine


def test_header_declares_the_api():
    names = engine.declared_symbols()
    for required in ("rp3dg_create", "rp3dg_destroy", "rp3dg_narrowphase_device", "rp3dg_narrowphase_host",
                     "rp3dg_create_convex_mesh", "rp3dg_create_convex_mesh_shape", "rp3dg_set_shapes"):
        assert required in names


def test_library_exports_every_declared_symbol(cuda_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", cuda_lib], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in engine.declared_symbols() if s not in exported]
    assert not missing, missing


def test_library_loads(cuda_lib):
    L = engine.load_library(cuda_lib)
    for s in engine.declared_symbols():
        assert hasattr(L, s)


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is None and
                    subprocess.run(["nvidia-smi"], capture_output=True).returncode == 0,
                    reason="a GPU is present")
def test_no_gpu_no_context(cuda_lib):
    L = engine.load_library(cuda_lib)
    h = C.c_void_p()
    assert L.rp3dg_create(0, C.byref(h)) == engine.RP3DG_ENODEV
    assert not h.value


def test_null_arguments_are_rejected(cuda_lib):
    L = engine.load_library(cuda_lib)
    assert L.rp3dg_narrowphase_device(None, 1, None, None, 1) == engine.RP3DG_EINVAL
    assert L.rp3dg_narrowphase_host(None, 1, None, None, 1) == engine.RP3DG_EINVAL
    assert L.rp3dg_set_shapes(None, None, 0) == engine.RP3DG_EINVAL
