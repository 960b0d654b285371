"""The C++ ReactorBase shim (include/pele/ReactorB200.H) compiles against a
stand-in for AMReX / PelePhysics (tests/cpp/ReactorBase.H), links the
library, registers under its factory name, and passes views that address
the same elements as the caller's Array4s.  Host only."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_shim_compiles_and_maps_array4(tmp_path):
    from pelelmex_b200 import build
    lib = build.build()
    exe = tmp_path / "shim_check"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", str(ROOT / "include"), "-I",
           str(ROOT / "tests" / "cpp"), str(ROOT / "tests" / "cpp" / "shim_check.cpp"), "-o", str(exe),
           "-L", str(lib.parent), "-lb200chem", f"-Wl,-rpath,{lib.parent}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    assert "shim ok" in run.stdout
