"""Build of the in-tree native libraries.

  op-pic_b200/lib/liboppb.so   CUDA kernels (sm_100a) + C ABI (include/oppb.h) and the
                               host set-up utilities (include/oppb_fempic.h)
  op-pic_b200/lib/libopp_b200.so  C++ drop-in runtime of the opp_* API (include/opp_lib.h)

Objects go to op-pic_b200/_build/.  A library is rebuilt when any of its sources or
headers is newer than it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
INC = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "lib"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{INC}"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", f"-I{INC}", "-Wall"]


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build command failed: {' '.join(cmd)}")


def build_oppb(force: bool = False) -> Path:
    """Compile csrc/*.cu and host/*.cpp into lib/liboppb.so."""
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    headers = sorted(INC.glob("*.h")) + sorted((PKG / "csrc").glob("*.cuh"))
    objs = []
    for src in sorted((PKG / "csrc").glob("*.cu")):
        obj = BUILD / (src.stem + ".cu.o")
        if force or _newer(obj, [src] + headers):
            _run([NVCC] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)])
        objs.append(obj)
    for src in sorted((PKG / "host").glob("*.cpp")):
        obj = BUILD / (src.stem + ".cpp.o")
        if force or _newer(obj, [src] + headers):
            _run(["g++"] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)])
        objs.append(obj)
    so = LIB / "liboppb.so"
    if force or _newer(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(so)] + [str(o) for o in objs])
    return so


def build_oracle(force: bool = False) -> Path:
    """Compile the C oracle (test infrastructure) into oracle/lib/liboppb_oracle.so."""
    src = ROOT / "oracle" / "fempic_oracle.c"
    out_dir = ROOT / "oracle" / "lib"
    out_dir.mkdir(exist_ok=True)
    so = out_dir / "liboppb_oracle.so"
    if force or _newer(so, [src]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-Wall", str(src), "-o", str(so)])
    return so


def build_reference(force: bool = False) -> bool:
    """Compile the reference seq/omp backends + harness into oracle/_ref (needs the
    reference sources; skipped when they are absent)."""
    if not Path("/root/reference/opp_lib").is_dir() or shutil.which("make") is None:
        return False
    if not (ROOT / "oracle" / "Makefile").exists():
        return False
    args = ["make", "-s", "-C", str(ROOT / "oracle"), "-j8"]
    if force:
        args.append("-B")
    _run(args)
    return True


def build_all(force: bool = False) -> None:
    build_oppb(force)
    build_oracle(force)
    build_reference(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", LIB / "liboppb.so")
