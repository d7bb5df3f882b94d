"""Randomised checks of the world step's host structures (no GPU): the pair
id maps against std::unordered_map, and the broad-phase tree code on a
trimmed device-style node span against the host tree
(tests/cpp/host_structures_fuzz.cpp, built with the host compiler)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_host_structures_fuzz(tmp_path):
    exe = str(tmp_path / "host_structures_fuzz")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", exe,
                    os.path.join(HERE, "cpp", "host_structures_fuzz.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "pair map 0 tree span 0" in r.stdout
