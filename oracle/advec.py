"""TEST INFRASTRUCTURE ONLY — Python driver of the NESO-advection oracle (advec_oracle.c) and
of the compiled reference harness (oracle/_ref/advec_ref_{seq,omp}); seq AoS layouts.
Only tests/ and bench.py's CPU legs may use it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle.oracle import load as _load_lib


def _lib() -> C.CDLL:
    lib = _load_lib()
    if not getattr(lib, "_advec_bound", False):
        vp, i32 = C.c_void_p, C.c_int32
        lib.oracle_advec_steps.restype = C.c_int
        lib.oracle_advec_steps.argtypes = [i32, vp, vp, vp, vp, vp, vp, C.c_double, vp, C.c_double, i32, i32,
                                           C.POINTER(C.c_int64)]
        lib._advec_bound = True
    return lib


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def steps(pos, vel, mdir, p2c, c2c, c_pos_ll, dt, extents, cell_width, n_steps, max_hops=1 << 20) -> int:
    """n_steps of update_pos + move over all particles, in place (pos [n,2] f64, vel [n,2],
    mdir [n,2] i32, p2c [n] i32, c2c [n_cells,4] i32, c_pos_ll [n_cells,2]).  Returns the
    move calls of the last step."""
    ext = np.ascontiguousarray(extents, dtype=np.float64)
    visits = C.c_int64(0)
    rc = _lib().oracle_advec_steps(len(p2c), _p(pos), _p(vel), _p(mdir), _p(p2c), _p(c2c), _p(c_pos_ll), dt,
                                   _p(ext), cell_width, n_steps, max_hops, C.byref(visits))
    if rc != 0:
        raise RuntimeError("oracle: a particle exceeded max_hops")
    return int(visits.value)


def steps_job(args) -> tuple:
    """One instance's n_steps in a worker process (args: pos, vel, mdir, p2c, c2c, c_pos_ll, dt,
    extents, cell_width, n_steps); returns (pos, mdir, p2c, move calls of the last step)."""
    pos, vel, mdir, p2c, c2c, c_pos_ll, dt, extents, cell_width, n_steps = args
    pos, mdir, p2c = pos.copy(), mdir.copy(), p2c.copy()
    v = steps(pos, vel, mdir, p2c, c2c, c_pos_ll, dt, extents, cell_width, n_steps)
    return pos, mdir, p2c, v


def run_reference(kind: str, nx, ny, cell_width, dt, pos, vel, mdir, p2c, c2c, c_pos_ll, n_steps,
                  threads: int | None = None) -> dict:
    """Run oracle/_ref/advec_ref_{seq,omp}: n_steps of update_pos + move.  Returns per-step wall
    times and the final pos, mdir, p2c."""
    import os
    import subprocess
    import tempfile
    from pathlib import Path

    from oracle.ref_runner import REF_DIR, params_text

    exe = REF_DIR / f"advec_ref_{kind}"
    if not exe.exists():
        raise FileNotFoundError(exe)
    n = len(p2c)
    hdr = np.zeros(1, dtype=[("magic", "S8"), ("ints", "<i4", 4), ("dbl", "<f8", 2)])
    hdr["magic"] = b"OPPBADV1"
    hdr["ints"] = [nx, ny, n, n_steps]
    hdr["dbl"] = [dt, cell_width]
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        with open(d / "case.bin", "wb") as f:
            f.write(hdr.tobytes())
            for a, t in ((c2c, "<i4"), (c_pos_ll, "<f8"), (pos, "<f8"), (vel, "<f8"), (mdir, "<i4"),
                         (p2c, "<i4")):
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

    ns = int(take("<i4", 1)[0])
    times = take("<f8", ns)
    size = int(take("<i4", 1)[0])
    return {"times": times, "pos": take("<f8", size * 2).reshape(size, 2), "mdir": take("<i4", size * 2).reshape(size, 2),
            "p2c": take("<i4", size)}
