"""TEST INFRASTRUCTURE ONLY — Python driver of the CabanaPIC oracle (cabana_oracle.c): the
move + current deposit of the generated seq backend, in its AoS host layout.
Only tests/ and bench.py's CPU legs may use it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle.oracle import load as _load_lib


def _lib() -> C.CDLL:
    lib = _load_lib()
    if not getattr(lib, "_cabana_bound", False):
        vp, i32 = C.c_void_p, C.c_int32
        lib.oracle_cabana_move_deposit.restype = C.c_int
        lib.oracle_cabana_move_deposit.argtypes = [i32, vp, vp, vp, vp, vp, vp, vp, vp, C.c_double, vp,
                                                   C.c_double, i32, C.POINTER(C.c_int64)]
        lib.oracle_cabana_move_deposit_mixed.restype = C.c_int
        lib.oracle_cabana_move_deposit_mixed.argtypes = lib.oracle_cabana_move_deposit.argtypes
        lib._cabana_bound = True
    return lib


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def move_deposit(pos, vel, streak, weight, p2c, c2ngc, interp, acc, qdt_2mc, cdt_d, qsp, max_hops=1 << 20):
    """opp_particle_move__move_deposit_kernel over all particles, in place.  Arrays: pos, vel,
    streak [n,3] f64; weight [n] f64; p2c [n] i32; c2ngc [n_cells,6] i32; interp [n_cells,18]
    f64; acc [n_cells,12] f64 (accumulated into).  Returns the number of kernel calls."""
    n = len(p2c)
    cd = np.ascontiguousarray(cdt_d, dtype=np.float64)
    visits = C.c_int64(0)
    rc = _lib().oracle_cabana_move_deposit(n, _p(pos), _p(vel), _p(streak), _p(weight), _p(p2c), _p(c2ngc),
                                           _p(interp), _p(acc), qdt_2mc, _p(cd), qsp, max_hops, C.byref(visits))
    if rc != 0:
        raise RuntimeError("oracle: a particle exceeded max_hops")
    return int(visits.value)


def move_deposit_mixed(pos, vel32, streak, weight, p2c, c2ngc, interp, acc, qdt_2mc, cdt_d, qsp, max_hops=1 << 20):
    """The FP32-momentum form (oracle_cabana_move_deposit_mixed): as move_deposit with vel32
    [n,3] FP32.  Returns the number of kernel calls."""
    n = len(p2c)
    cd = np.ascontiguousarray(cdt_d, dtype=np.float64)
    visits = C.c_int64(0)
    rc = _lib().oracle_cabana_move_deposit_mixed(n, _p(pos), _p(vel32), _p(streak), _p(weight), _p(p2c), _p(c2ngc),
                                                 _p(interp), _p(acc), qdt_2mc, _p(cd), qsp, max_hops, C.byref(visits))
    if rc != 0:
        raise RuntimeError("oracle: a particle exceeded max_hops")
    return int(visits.value)


def run_reference(kind: str, c2ngc, interp, pos, vel, streak, weight, p2c, qdt_2mc, cdt_d, qsp, dt=0.0,
                  calls: int = 1, threads: int | None = None) -> dict:
    """Run the compiled reference (oracle/_ref/cabana_ref_{seq,omp}) on the case: `calls`
    times opp_reset_dat(c_acc) + opp_particle_move__move_deposit_kernel with fixed c_interp.
    Returns the per-call wall times, the final particle dats and the last call's c_acc."""
    import os
    import subprocess
    import tempfile
    from pathlib import Path

    from oracle.ref_runner import REF_DIR, params_text

    exe = REF_DIR / f"cabana_ref_{kind}"
    if not exe.exists():
        raise FileNotFoundError(exe)
    nc, n = len(c2ngc), len(p2c)
    hdr = np.zeros(1, dtype=[("magic", "S8"), ("ints", "<i4", 4), ("dbl", "<f8", 6)])
    hdr["magic"] = b"OPPBCAB1"
    hdr["ints"] = [nc, n, calls, 0]
    hdr["dbl"] = [qdt_2mc, cdt_d[0], cdt_d[1], cdt_d[2], qsp, dt]
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        with open(d / "case.bin", "wb") as f:
            f.write(hdr.tobytes())
            for a, t in ((c2ngc, "<i4"), (interp, "<f8"), (pos, "<f8"), (vel, "<f8"), (streak, "<f8"),
                         (weight, "<f8"), (p2c, "<i4")):
                f.write(np.ascontiguousarray(a, dtype=t).tobytes())
        (d / "params.txt").write_text(params_text("HoleFill_All", 10, 2.0))
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        r = subprocess.run([str(exe), str(d / "params.txt"), str(d / "case.bin"), str(d / "out.bin")],
                           capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"{exe.name} failed ({r.returncode}): {r.stderr[-2000:]}")
        raw = (d / "out.bin").read_bytes()
    off = 0

    def take(dt_, count):
        nonlocal off
        a = np.frombuffer(raw[off:off + count * np.dtype(dt_).itemsize], dt_).copy()
        off += count * np.dtype(dt_).itemsize
        return a

    ncalls = int(take("<i4", 1)[0])
    times = take("<f8", ncalls)
    size = int(take("<i4", 1)[0])
    return {"times": times, "pos": take("<f8", size * 3).reshape(size, 3), "vel": take("<f8", size * 3).reshape(size, 3),
            "streak": take("<f8", size * 3).reshape(size, 3), "p2c": take("<i4", size),
            "acc": take("<f8", nc * 12).reshape(nc, 12)}
