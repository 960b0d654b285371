"""Build the in-tree CUDA library libb200chem.so for sm_100a.

    python -m pelelmex_b200.build [--force]

nvcc cross-compiles without a GPU.  The library is rebuilt only when a
source under csrc/ or include/ is newer than it.
"""
from __future__ import annotations

import argparse
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libb200chem.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-diag-suppress", "128"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def write_generated(gendir: Path) -> Path:
    """Mechanism-specific right-hand sides of the bundled mechanisms
    (pelelmex_b200.mechgen); the file is rewritten only when it changes."""
    sys.path.insert(0, str(ROOT))
    from pelelmex_b200 import mechgen
    gendir.mkdir(parents=True, exist_ok=True)
    path = gendir / "gen_mechs.cuh"
    text = mechgen.generate_bundled()
    if not path.exists() or path.read_text() != text:
        path.write_text(text)
    return path


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False, jobs: int = 0) -> Path:
    """Compile every csrc/*.cu to an object in parallel, then link libb200chem.so."""
    import concurrent.futures as cf
    import os

    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    gen = write_generated(objdir / "gen")
    deps = list(CSRC.glob("*")) + list(INCLUDE.rglob("*.h")) + list(INCLUDE.rglob("*.H")) + [gen]
    if not force and not _stale(LIB, deps):
        return LIB
    srcs = sources()

    def compile_one(src: Path):
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", "-o", str(obj), str(src), "-I", str(INCLUDE), "-I",
               str(gen.parent)]
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
        return src, obj, cmd, subprocess.run(cmd, capture_output=True, text=True)

    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    objs, logs = [], []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for src, obj, cmd, res in ex.map(compile_one, srcs):
            if verbose:
                print(" ".join(cmd), flush=True)
            if res.returncode != 0:
                sys.stderr.write(res.stdout + res.stderr)
                raise RuntimeError(f"nvcc failed on {src.name}")
            logs.append(res.stderr)
            objs.append(str(obj))
    res = subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *objs], capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("linking libb200chem.so failed")
    if verbose or ptxas_v:
        sys.stderr.write("".join(logs))
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True, ptxas_v=a.ptxas_v))


if __name__ == "__main__":
    main()
