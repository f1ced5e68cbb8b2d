"""In-tree build of the native libraries (no setup.py, no JIT cache).

Outputs, all inside the package so they travel with the repository snapshot:

* ``lib/libwgpauli.so``   sm_100a CUDA kernels + the wg_* C-ABI (include/wg_pauli.h)
* ``lib/libwolfgang.so``  the C++ drop-in classes (include/wolfgang/*.hpp)
* ``_wolfgang_core*.so``  the Python module (pybind11)

Every CUDA translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``.  Host code is compiled
with ``-ffp-contract=off`` so host-side floating point matches the reference's
g++ -O2 build.  Rebuilds are incremental (by modification time).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = CSRC / "host"
LIB = PKG / "lib"
OBJ = PKG / "_build"
INCLUDE = ROOT / "include"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
CXX = os.environ.get("CXX", "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-I", str(INCLUDE), "-I", str(CSRC),
]
CXX_FLAGS = ["-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-Wall",
             "-I", str(INCLUDE), "-I", str(HOST)]

# Shared libraries link libstdc++ as the shared system library, named
# explicitly: a toolchain whose libstdc++.so link is dangling falls back to
# libstdc++.a, and the copy it links in exports unique symbols (the old
# std::string's empty representation among them) that libraries loaded later
# in the same process bind to, so that they free memory of the wrong copy
# (torch's import crashed after this package's).  --exclude-libs hides
# anything still taken from a static archive.
SHARED_LINK = ["-l:libstdc++.so.6", "-Wl,--exclude-libs,ALL"]

CU_SOURCES = ["wg_runtime.cu", "wg_commute.cu", "wg_simplify.cu", "wg_bucket.cu", "wg_expect.cu", "wg_group.cu",
              "wg_batch.cu", "wg_tune.cu"]
CU_HEADERS = ["wg_common.cuh", "wg_scan.cuh"]
HOST_SOURCES = ["pauli_sum.cpp", "device.cpp"]
HOST_HEADERS = ["abi.hpp", "guards.hpp"]


def _ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


def module_path() -> Path:
    return PKG / ("_wolfgang_core" + _ext_suffix())


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}")


def _common_deps() -> list[Path]:
    return [CSRC / h for h in CU_HEADERS] + [INCLUDE / "wg_pauli.h"]


def _dlpack_include() -> str:
    """Directory holding ATen/dlpack.h, the DLPack C ABI header that torch
    ships (a standalone C header; the module includes nothing else of torch)."""
    import importlib.util

    spec = importlib.util.find_spec("torch")
    if spec is None or not spec.submodule_search_locations:
        raise RuntimeError("torch's include directory (for ATen/dlpack.h) was not found")
    inc = Path(list(spec.submodule_search_locations)[0]) / "include"
    if not (inc / "ATen" / "dlpack.h").exists():
        raise RuntimeError(f"ATen/dlpack.h not found under {inc}")
    return str(inc)


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile everything that is out of date; return the Python module path."""
    if not Path(NVCC).exists() and shutil.which("nvcc") is None:
        raise RuntimeError("nvcc not found: set CUDA_HOME")
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    jobs = jobs or min(8, os.cpu_count() or 4)

    # 1. CUDA objects -> libwgpauli.so
    cu_jobs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = OBJ / (s.stem + ".o")
        if _stale(o, [s] + _common_deps()):
            cu_jobs.append([NVCC, *NVCC_FLAGS, "-c", str(s), "-o", str(o)])
    with ThreadPoolExecutor(jobs) as ex:
        list(ex.map(_run, cu_jobs))
    wgpauli = LIB / "libwgpauli.so"
    cu_objs = [OBJ / (Path(s).stem + ".o") for s in CU_SOURCES]
    if _stale(wgpauli, cu_objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(wgpauli), *map(str, cu_objs)])

    # 2. C++ drop-in classes -> libwolfgang.so
    host_deps = [HOST / h for h in HOST_HEADERS] + list((INCLUDE / "wolfgang").glob("*.hpp")) + [INCLUDE / "wg_pauli.h"]
    host_jobs = []
    for src in HOST_SOURCES:
        s = HOST / src
        o = OBJ / ("host_" + s.stem + ".o")
        if _stale(o, [s] + host_deps):
            host_jobs.append([CXX, *CXX_FLAGS, "-c", str(s), "-o", str(o)])
    with ThreadPoolExecutor(jobs) as ex:
        list(ex.map(_run, host_jobs))
    wolfgang = LIB / "libwolfgang.so"
    host_objs = [OBJ / ("host_" + Path(s).stem + ".o") for s in HOST_SOURCES]
    if _stale(wolfgang, host_objs + [wgpauli]):
        _run([CXX, "-shared", "-o", str(wolfgang), *map(str, host_objs), f"-L{LIB}", "-lwgpauli",
              "-Wl,-rpath,$ORIGIN", *SHARED_LINK])

    # 3. Python module
    import pybind11

    mod = module_path()
    msrc = HOST / "module.cpp"
    if _stale(mod, [msrc, wolfgang] + host_deps):
        _run([CXX, *CXX_FLAGS, "-shared", "-o", str(mod), str(msrc),
              "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"], "-I", _dlpack_include(),
              f"-L{LIB}", "-lwolfgang", "-lwgpauli", "-Wl,-rpath,$ORIGIN/lib", *SHARED_LINK])
    if verbose:
        print(f"built {wgpauli}, {wolfgang}, {mod}")
    return mod


def ptxas_report() -> str:
    """Register / spill / shared-memory report of every kernel (-Xptxas -v)."""
    out = []
    for src in CU_SOURCES:
        proc = subprocess.run([NVCC, *NVCC_FLAGS, "-Xptxas", "-v", "-c", str(CSRC / src), "-o", os.devnull],
                              stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        out.append(proc.stdout)
    return "\n".join(out)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--ptxas":
        print(ptxas_report())
    else:
        build(verbose=True)
