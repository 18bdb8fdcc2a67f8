"""Build the engine's shared library in-tree with nvcc for sm_100a.

    python -m cudagravitydemo_b200.build          # libbh_b200.so next to this file

Sources: csrc/*.cu (kernels + C ABI) and host/*.c (seeded initial
conditions).  Objects go to _build/; a source is recompiled when it or any
header is newer than its object.  Then the C simulation program
driver/gravity_sim.c is compiled with gcc against the library (gravity_sim
next to it, found at run time through an $ORIGIN rpath).
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
INCLUDE = ROOT / "include"
CSRC = PKG / "csrc"
HOST = PKG / "host"
BUILD = PKG / "_build"
LIB = PKG / "libbh_b200.so"
DRIVER_SRC = PKG / "driver" / "gravity_sim.c"
DRIVER = PKG / "gravity_sim"
CUDA_INCLUDE = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xcompiler", "-Wall"]
CC_FLAGS = ["-O2", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libbh_b200.so")
    return path


def _headers() -> list[Path]:
    return sorted(INCLUDE.glob("*.h")) + sorted(CSRC.glob("*.cuh"))


def _stale(obj: Path, src: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    flags = NVCC_FLAGS if src.suffix == ".cu" else CC_FLAGS
    cmd = [nvcc(), *ARCH, *flags, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(HOST.glob("*.c"))
    newest = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    objs = []
    for src in sources:
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, src, newest):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(lambda j: _compile(j[0], j[1], verbose), jobs))
    if jobs or not LIB.exists() or force:
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-lpthread",
               "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking libbh_b200.so failed:\n{r.stdout}\n{r.stderr}")
    build_driver(verbose, force)
    return LIB


def build_driver(verbose: bool = False, force: bool = False) -> Path:
    """gcc the C simulation program against libbh_b200.so."""
    newest = max([DRIVER_SRC.stat().st_mtime, LIB.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if not force and DRIVER.exists() and DRIVER.stat().st_mtime >= newest:
        return DRIVER
    cc = shutil.which("gcc") or "cc"
    cmd = [cc, "-O2", "-Wall", "-std=c11", "-D_POSIX_C_SOURCE=199309L", "-I", str(INCLUDE), "-I", str(CUDA_INCLUDE),
           str(DRIVER_SRC), "-o", str(DRIVER), "-L", str(PKG), "-lbh_b200", "-lm", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building gravity_sim failed:\n{r.stdout}\n{r.stderr}")
    return DRIVER


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
