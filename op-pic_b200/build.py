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
# Sources whose FP64 expressions must keep the reference's written order with one rounding
# per operation: no FMA contraction anywhere in the file.
PER_FILE_NVCC_FLAGS = {"cabana.cu": ["-fmad=false"], "cabana_field.cu": ["-fmad=false"], "advec.cu": ["-fmad=false"],
                       "field.cu": ["-fmad=false"],
                       # the grid set-up loops of the direct-hop mapper run on the host
                       "dh.cu": ["-Xcompiler", "-ffp-contract=off"]}


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


CUDA_INC = "/usr/local/cuda/include"
# Host sources of the C ABI library (set-up utilities) and of the C++ drop-in runtime.
ABI_HOST = ("fempic_mesh.cpp", "fempic_field.cpp")
RUNTIME_HOST = ("fempic_mesh.cpp", "fempic_field.cpp", "opp_runtime.cpp", "fempic_loops.cpp", "fempic_field_solver.cpp",
                "advec_loops.cpp", "cabana_loops.cpp")


def _objects(force: bool, names) -> list[Path]:
    BUILD.mkdir(exist_ok=True)
    headers = sorted(INC.glob("*.h")) + sorted((PKG / "csrc").glob("*.cuh"))
    objs = []
    for src in sorted((PKG / "csrc").glob("*.cu")):
        obj = BUILD / (src.stem + ".cu.o")
        if force or _newer(obj, [src] + headers):
            _run([NVCC] + NVCC_FLAGS + PER_FILE_NVCC_FLAGS.get(src.name, []) + ["-c", str(src), "-o", str(obj)])
        objs.append(obj)
    for name in names:
        src = PKG / "host" / name
        obj = BUILD / (src.stem + ".cpp.o")
        if force or _newer(obj, [src] + headers):
            _run(["g++"] + CXX_FLAGS + [f"-I{CUDA_INC}", "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    return objs


def build_oppb(force: bool = False) -> Path:
    """Compile csrc/*.cu and the set-up utilities into lib/liboppb.so (the C ABI), and
    the same kernels with the opp_* runtime into lib/libopp_b200.so (the C++ drop-in),
    plus the FemPIC app linked against the latter."""
    LIB.mkdir(exist_ok=True)
    objs = _objects(force, ABI_HOST)
    so = LIB / "liboppb.so"
    if force or _newer(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(so)] + [str(o) for o in objs])
    robjs = _objects(False, RUNTIME_HOST)
    rso = LIB / "libopp_b200.so"
    if force or _newer(rso, robjs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(rso)] + [str(o) for o in robjs])
    app_src = PKG / "apps" / "fempic" / "fempic_b200.cpp"
    app = LIB / "fempic_b200"
    if force or _newer(app, [app_src, rso] + sorted(INC.glob("*.h"))):
        _run(["g++"] + CXX_FLAGS + [f"-I{CUDA_INC}", str(app_src), "-o", str(app), f"-L{LIB}", "-lopp_b200",
                                    "-Wl,-rpath,$ORIGIN"])
    return so


def build_oracle(force: bool = False) -> Path:
    """Compile the C oracle (test infrastructure) into oracle/lib/liboppb_oracle.so."""
    srcs = [ROOT / "oracle" / "fempic_oracle.c", ROOT / "oracle" / "cabana_oracle.c", ROOT / "oracle" / "advec_oracle.c",
            ROOT / "oracle" / "field_oracle.c"]
    out_dir = ROOT / "oracle" / "lib"
    out_dir.mkdir(exist_ok=True)
    so = out_dir / "liboppb_oracle.so"
    if force or _newer(so, srcs):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-Wall", *map(str, srcs),
              "-o", str(so), "-lm"])
    return so


def reference_dir() -> Path:
    """Root of the OP-PIC source tree: the OPPB_REFERENCE_DIR environment variable, else a
    `reference` directory beside this repository."""
    env = os.environ.get("OPPB_REFERENCE_DIR")
    return Path(env) if env else ROOT.parent / "reference"


def build_reference(force: bool = False) -> bool:
    """Compile the reference seq/omp backends + harness into oracle/_ref (needs the
    reference sources; skipped when they are absent)."""
    ref = reference_dir()
    if not (ref / "opp_lib").is_dir() or shutil.which("make") is None:
        return False
    if not (ROOT / "oracle" / "Makefile").exists():
        return False
    args = ["make", "-s", "-C", str(ROOT / "oracle"), "-j8", f"REF={ref}"]
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
