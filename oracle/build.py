"""Build recipe for the test oracle (TEST INFRASTRUCTURE ONLY).

    python -m oracle.build

1. oracle/_build/liboracle.so — the C restatement (bh_oracle.c), compiled
   with -ffp-contract=off so no multiply-add is fused except the explicit
   fmaf() calls that mirror nvcc's contractions in the reference, plus the
   seeded initial-condition generators (host/ics.c) for inputs made without
   the engine library.
2. oracle/_ref/libref.so — the reference itself: its own sources, compiled
   from where they lie under the reference checkout, for sm_100a with the
   reference makefile's release options (makefile:5-27; -march=native is left
   out so the library runs on any x86-64 host) plus -Dmain=ref_main, two
   stand-in headers for files the reference includes but does not ship
   (ref_stubs/CPUTree.h, ref_stubs/cglm/cglm.h) and ref_harness.cu, which
   drives the reference's step on given inputs.  Built only when the reference
   checkout is present; the prebuilt library travels with the repository.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
# The reference checkout: $BH_REFERENCE_DIR, else a directory named
# "reference" beside this repository.  Absent (as on a machine that only runs
# the tests), the prebuilt oracle/_ref/libref.so is used as it is.
REFERENCE = Path(os.environ.get("BH_REFERENCE_DIR") or (ROOT.parent / "reference"))
ORACLE_LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref.so"

REF_SOURCES = ["basicGravity.cu", "tree.cu", "sorting.cu", "units.c", "inputOutput.c", "initialConditions.c"]


def _run(cmd: list[str], what: str) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{what} failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_oracle(force: bool = False) -> Path:
    src = HERE / "bh_oracle.c"
    # the seeded initial-condition generators, so that the CPU baselines and
    # the reference arm make their inputs without loading the engine library
    ics = ROOT / "cudagravitydemo_b200" / "host" / "ics.c"
    hdrs = [HERE / "bh_oracle.h", ROOT / "include" / "types.h", ROOT / "include" / "bh_api.h"]
    if not force and ORACLE_LIB.exists() and all(ORACLE_LIB.stat().st_mtime >= p.stat().st_mtime
                                                  for p in [src, ics, *hdrs, Path(__file__)]):
        return ORACLE_LIB
    ORACLE_LIB.parent.mkdir(exist_ok=True)
    cuda_inc = Path(shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc").resolve().parent.parent / "include"
    _run(["gcc", "-O3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fno-math-errno", "-fPIC", "-shared",
          "-Wall",
          f"-I{ROOT / 'include'}", f"-I{cuda_inc}", str(src), str(ics), "-o", str(ORACLE_LIB), "-lm"],
         "oracle build")
    return ORACLE_LIB


def build_reference(force: bool = False) -> Path | None:
    if not all((REFERENCE / s).exists() for s in REF_SOURCES):
        return REF_LIB if REF_LIB.exists() else None
    inputs = [REFERENCE / s for s in REF_SOURCES] + [HERE / "ref_harness.cu", HERE / "build.py"]
    if not force and REF_LIB.exists() and all(REF_LIB.stat().st_mtime >= p.stat().st_mtime for p in inputs):
        return REF_LIB
    REF_LIB.parent.mkdir(exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O3", "-Xcompiler=-ffast-math",
           "-Xcompiler=-fPIC", "-shared", "-Dmain=ref_main", f"-I{HERE / 'ref_stubs'}", f"-I{REFERENCE}",
           *[str(REFERENCE / s) for s in REF_SOURCES], str(HERE / "ref_harness.cu"),
           "-Xlinker", "-Bsymbolic", "-o", str(REF_LIB)]
    _run(cmd, "reference build")
    return REF_LIB


def build(force: bool = False) -> None:
    build_oracle(force)
    build_reference(force)


if __name__ == "__main__":
    build(force="-f" in sys.argv)
    print(ORACLE_LIB, REF_LIB if REF_LIB.exists() else "(reference not built)")
