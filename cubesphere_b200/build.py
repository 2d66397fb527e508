"""In-tree build of the CUDA library (sm_100a) and of the CPU oracle.

``python -m cubesphere_b200.build`` compiles

* ``cubesphere_b200/libcubesphere_b200.so`` from ``cubesphere_b200/csrc``
  (CUDA kernels for ``sm_100a`` + the host mesh builder and C ABI), and
* ``oracle/liboracle.so`` (the CPU restatement used only by the tests,
  ``__graft_entry__.smoke`` and the CPU baseline of ``bench.py``).

Objects are rebuilt only when a source or header is newer than them.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "cubesphere_b200"
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcubesphere_b200.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp",
              "-I", str(ROOT / "include")] + ARCH
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-I", str(ROOT / "include")]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_library(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    jobs = []
    objs = []
    for src in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not _stale(obj, [src] + headers):
            continue
        if src.suffix == ".cu":
            cmd = [NVCC] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)]
        jobs.append(cmd)
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd), flush=True)
        list(ex.map(_run, jobs))
    if _stale(LIB, objs):
        _run([NVCC, "-shared"] + ARCH + ["-o", str(LIB)] + [str(o) for o in objs] + ["-Xcompiler", "-fopenmp", "-lgomp"])
    return LIB


def build_oracle() -> Path:
    """The oracle library: oracle.cpp plus the host mesh builder and seeded
    initial state compiled from their sources (mesh.cpp, init.cpp), so that
    a CPU solve loads nothing else."""
    srcs = [ORACLE_DIR / "oracle.cpp", CSRC / "mesh.cpp", CSRC / "init.cpp"]
    deps = srcs + [ORACLE_DIR / "oracle_core.h", CSRC / "cs_internal.h", ROOT / "include" / "cubesphere_b200.h"]
    if _stale(ORACLE_LIB, deps):
        # No FMA contraction: the oracle evaluates every expression as written.
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp",
              "-I", str(ROOT / "include"), "-I", str(CSRC), "-o", str(ORACLE_LIB)] + [str(s) for s in srcs])
    return ORACLE_LIB


def main() -> int:
    verbose = "-v" in sys.argv
    print(build_library(verbose))
    print(build_oracle())
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
