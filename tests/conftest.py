import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_port_oracle():
    lib = os.path.join(ROOT, "oracle", "librp3d_oracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       stdout=subprocess.DEVNULL)
    return lib


@pytest.fixture(scope="session")
def port():
    _ensure_port_oracle()
    import reflib
    return reflib.PortEngine()


@pytest.fixture(scope="session")
def cuda_lib():
    """Path of librp3dg.so, built in-tree if it is missing."""
    from reactphysics3d_b200 import build, engine
    if not os.path.exists(engine.LIB_PATH):
        build.build()
    return engine.LIB_PATH
