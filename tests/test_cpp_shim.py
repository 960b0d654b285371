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


def _compile_react(tmp_path, mech_name):
    from pelelmex_b200 import build, mechanism as M, mechgen
    lib = build.build()
    md = tmp_path / "mech_desc.cpp"
    md.write_text(mechgen.generate_mech_desc(M.flatten(M.builtin(mech_name)), mech_name))
    exe = tmp_path / "shim_react"
    cuda = Path("/usr/local/cuda")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-I", str(ROOT / "include"), "-I", str(ROOT / "tests" / "cpp"), "-I",
           str(cuda / "include"), str(ROOT / "tests" / "cpp" / "shim_react.cpp"), str(md), "-o", str(exe), "-L",
           str(lib.parent), "-lb200chem", "-L", str(cuda / "lib64"), "-lcudart", f"-Wl,-rpath,{lib.parent}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def _run_react(tmp_path, exe, f, dims, ghost, weights=None):
    import numpy as np
    N = f.rhoY.shape[0]
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as fh:
        fh.write(np.array([N, *dims, ghost], np.int32).tobytes())
        fh.write(np.array([f.dt], np.float64).tobytes())
        for a in (f.rhoY, f.T, f.rhoH):
            fh.write(np.ascontiguousarray(a, np.float64).tobytes())
    args = [str(exe), str(inp), str(out)] + ([str(weights)] if weights else [])
    run = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr
    raw = np.fromfile(out, dtype=np.float64, count=(N + 3) * f.ncells)
    hybrid = int(np.fromfile(out, dtype=np.int32, offset=8 * (N + 3) * f.ncells)[0])
    c = f.ncells
    return raw[:N * c].reshape(N, c), raw[N * c:(N + 1) * c], raw[(N + 1) * c:(N + 2) * c], raw[(N + 2) * c:], hybrid


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_shim_reacts_device_fabs_like_the_oracle(tmp_path):
    """ReactorBase::create("ReactorB200") -> init -> set_eos_parm -> react on
    device Array4 fabs with ghost cells (a 4 x 4 x 4 box of the LiDryer-shaped
    case), mechanism from the generated b200chem_make_mech_desc(): the oracle's
    result within the parity tolerances, ghost cells untouched."""
    import numpy as np
    import oracle
    from pelelmex_b200 import mechanism as M, workloads as W
    mech = M.builtin("synth_h2_9")
    f = W.premixed_h2(mech, edge=4)
    exe = _compile_react(tmp_path, "synth_h2_9")
    rY, T, rH, fc, hybrid = _run_react(tmp_path, exe, f, (4, 4, 4), 2)
    ref = oracle.Oracle(M.flatten(mech)).react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-8, atol=1e-12,
                                               max_order=5)
    rho = f.rhoY.sum(axis=0)
    assert hybrid == 0
    assert np.max(np.abs(T - ref["T"]) / ref["T"]) <= 1e-5
    assert np.max(np.abs(rY - ref["rhoY"]) / rho) <= 1e-8
    assert np.array_equal(rH, f.rhoH)  # no enthalpy forcing
    assert (fc > 0).all()


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_shim_selects_the_hybrid_from_the_inputs_key(tmp_path):
    """b200.surrogate = <weights file> selects the surrogate-first react: on an
    8 x 8 x 8 box of held-out flame cells every cell stays within the 1e-4
    relative T bar of the oracle and some cells are taken by the surrogate
    (fctCount 0)."""
    import numpy as np
    import oracle
    from pelelmex_b200 import mechanism as M, workloads as W
    weights = ROOT / "pelelmex_b200" / "surrogates" / "synth_ch4_21.b2s"
    mech = M.builtin("synth_ch4_21")
    f = W.flame_ch4(mech, cells=W.sample_cells(128 ** 3, 512, seed=55), seed=5, dt=1e-6)
    exe = _compile_react(tmp_path, "synth_ch4_21")
    rY, T, rH, fc, hybrid = _run_react(tmp_path, exe, f, (8, 8, 8), 1, weights)
    ref = oracle.Oracle(M.flatten(mech)).react(f.rhoY, f.frhoY, f.T, f.rhoH, f.frhoH, f.dt, rtol=1e-8, atol=1e-12,
                                               max_order=5)
    assert hybrid == 1
    assert np.max(np.abs(T - ref["T"]) / ref["T"]) <= 1e-4
    assert (fc == 0).sum() > 0 and (fc > 0).sum() > 0
