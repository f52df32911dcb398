"""In-tree build of the native parts.

* ``openstc_b200/libopenstc_b200.so`` - the C ABI (include/openstc_b200.h):
  host C++ (case reader, mesh, driver) compiled with g++, sm_100a kernels
  compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a``.
* ``openstc_b200/bin/openstc`` - the command-line driver.
* ``oracle/libostc_oracle.so`` - the CPU oracle used by the tests and the CPU
  baseline (built here because the build check compiles every native part;
  the library itself never links it).

Objects are rebuilt when a source or any header under csrc/ is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libopenstc_b200.so"
BIN = PKG / "bin" / "openstc"
ORACLE_SRC = ROOT / "oracle" / "ostc_oracle.c"
ORACLE_LIB = ROOT / "oracle" / "libostc_oracle.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++20", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++20", "-fPIC", "-Wall", "-Wno-unused-function"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_home() -> Path:
    return Path(_nvcc()).resolve().parent.parent


def _newest_header() -> float:
    stamps = [p.stat().st_mtime for p in CSRC.rglob("*") if p.suffix in (".hpp", ".cuh", ".h")]
    stamps.append((ROOT / "include" / "openstc_b200.h").stat().st_mtime)
    return max(stamps)


def _stale(obj: Path, src: Path, hdr: float) -> bool:
    return not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build step failed ({res.returncode}):\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def build_oracle(verbose: bool = False) -> Path:
    if ORACLE_LIB.exists() and ORACLE_LIB.stat().st_mtime >= max(
        ORACLE_SRC.stat().st_mtime, (ROOT / "oracle" / "ostc_oracle.h").stat().st_mtime
    ):
        return ORACLE_LIB
    _run(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11", str(ORACLE_SRC), "-o", str(ORACLE_LIB), "-lm"],
         verbose)
    return ORACLE_LIB


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile everything that is out of date; returns the library path."""
    BUILD.mkdir(exist_ok=True)
    (PKG / "bin").mkdir(exist_ok=True)
    hdr = _newest_header()
    nvcc = _nvcc()
    inc = ["-I", str(ROOT / "include"), "-I", str(CSRC)]
    cuda_inc = ["-I", str(_cuda_home() / "include")]
    jobs_ = []
    objs = []
    for src in sorted((CSRC / "host").glob("*.cpp")) + [CSRC / "capi.cpp"]:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if _stale(obj, src, hdr):
            jobs_.append(["g++", *CXX_FLAGS, *inc, *cuda_inc, "-c", str(src), "-o", str(obj)])
    for src in sorted((CSRC / "device").glob("*.cu")):
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if _stale(obj, src, hdr):
            jobs_.append([nvcc, *NVCC_FLAGS, *inc, "-c", str(src), "-o", str(obj)])
    main_obj = BUILD / "main.o"
    if _stale(main_obj, CSRC / "main.cpp", hdr):
        jobs_.append(["g++", *CXX_FLAGS, *inc, *cuda_inc, "-c", str(CSRC / "main.cpp"), "-o", str(main_obj)])
    workers = jobs or max(1, min(len(jobs_), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(max_workers=max(1, workers)) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs_))
    newest_obj = max(o.stat().st_mtime for o in objs)
    if jobs_ or not LIB.exists() or LIB.stat().st_mtime < newest_obj:
        _run([nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", *[str(o) for o in objs], "-o", str(LIB)], verbose)
    if jobs_ or not BIN.exists() or BIN.stat().st_mtime < newest_obj:
        _run([nvcc, *ARCH, str(main_obj), *[str(o) for o in objs if o.name != "capi.o"], "-o", str(BIN)], verbose)
    build_oracle(verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
