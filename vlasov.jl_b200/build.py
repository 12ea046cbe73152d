"""Builds the native parts in-tree.

* ``vlasov.jl_b200/lib/libvlasov_b200.so`` -- the CUDA library (sm_100a) with
  the C ABI of ``include/vlasov_b200.h``;
* ``oracle/liboracle.so`` -- the float64 CPU oracle (test infrastructure).

Both are plain compiler invocations (nvcc / g++), rebuilt when a source is
newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libvlasov_b200.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--shared", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA library cannot be built")


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """One object per source, compiled in parallel, then one link."""
    headers = sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "vlasov_b200.h"]
    deps = _sources() + headers
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = LIBDIR / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "--shared"]
    jobs = []
    for src in _sources():
        obj = objdir / (src.name + ".o")
        if force or _stale(obj, [src, *headers]):
            jobs.append([_nvcc(), *ARCH, *compile_flags, "-I", str(ROOT / "include"), "-c", str(src),
                         "-o", str(obj)])
    if verbose:
        for cmd in jobs:
            print(" ".join(cmd), file=sys.stderr)
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4) or 1) as pool:
        done = list(pool.map(lambda cmd: subprocess.run(cmd, capture_output=True, text=True), jobs))
    for cmd, r in zip(jobs, done):
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise subprocess.CalledProcessError(r.returncode, cmd)
    link = [_nvcc(), *ARCH, "--shared", "-Xcompiler", "-fPIC",
            *[str(objdir / (src.name + ".o")) for src in _sources()], "-o", str(LIB), "-lcudart"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    return LIB


def build_oracle(force: bool = False, verbose: bool = False) -> Path:
    src = ORACLE_DIR / "vlasov_oracle.cpp"
    if not force and not _stale(ORACLE_LIB, [src]):
        return ORACLE_LIB
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-ffp-contract=off", "-shared", "-fPIC",
           "-std=c++17", str(src), "-o", str(ORACLE_LIB)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return ORACLE_LIB


def build_all(force: bool = False, verbose: bool = False):
    return build_library(force, verbose), build_oracle(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
