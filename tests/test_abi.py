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


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return subprocess.run(["nvidia-smi"], capture_output=True).returncode == 0


@pytest.mark.skipif(_gpu_present(), reason="a GPU is present")
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


def test_struct_layouts_match_the_python_dtypes(tmp_path):
    """The public structs as a C compiler lays them out from include/rp3dg.h
    (sizes and field offsets) are the numpy dtypes the Python side uses."""
    import shutil
    import subprocess

    import numpy as np

    from reactphysics3d_b200 import _abi as A
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"rp3dg_joint_desc": A.JOINT_DESC_DTYPE, "rp3dg_ray": A.RAY_DTYPE,
               "rp3dg_raycast_hit": A.RAYCAST_HIT_DTYPE, "rp3dg_contact_event": A.CONTACT_EVENT_DTYPE,
               "rp3dg_world_settings": A.WORLD_SETTINGS_DTYPE, "rp3dg_body_desc": A.BODY_DESC_DTYPE,
               "rp3dg_collider_desc": A.COLLIDER_DESC_DTYPE, "rp3dg_world_stats": A.WORLD_STATS_DTYPE}
    # ctypes structures of the bindings, as (size, {field: offset})
    from reactphysics3d_b200 import broadphase as BP
    ctypes_structs = {"rp3dg_solver_stats": engine.SolverStats, "rp3dg_broadphase": BP.BroadPhase}
    layouts = {name: (dt.itemsize, {f: dt.fields[f][1] for f in dt.names}) for name, dt in structs.items()}
    layouts.update({name: (C.sizeof(st), {f: getattr(st, f).offset for f, _ in st._fields_})
                    for name, st in ctypes_structs.items()})
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{os.path.join(root, "include", "rp3dg.h")}"',
             "int main(void) {"]
    for name, (size, fields) in layouts.items():
        lines.append(f'    printf("{name} %zu\\n", sizeof({name}));')
        for f in fields:
            lines.append(f'    printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, str(src), "-o", str(exe)], check=True)
    got = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                          check=True).stdout.splitlines())
    for name, (size, fields) in layouts.items():
        assert int(got[name]) == size, name
        for f, off in fields.items():
            assert int(got[f"{name}.{f}"]) == off, (name, f)
