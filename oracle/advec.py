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
        lib.oracle_advec_steps_dh.restype = C.c_int
        lib.oracle_advec_steps_dh.argtypes = [i32, vp, vp, vp, vp, vp, vp, C.c_double, vp, C.c_double, i32, i32,
                                              vp, vp, C.c_double, vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.oracle_advec_move_dh.restype = C.c_int
        lib.oracle_advec_move_dh.argtypes = [i32, vp, vp, vp, vp, vp, vp, C.c_double, i32, vp, vp, C.c_double, vp,
                                             C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.oracle_advec_dh_grid_init.restype = C.c_int
        lib.oracle_advec_dh_grid_init.argtypes = [i32, vp, C.c_double, vp, vp, vp]
        lib.oracle_advec_dh_build.restype = None
        lib.oracle_advec_dh_build.argtypes = [i32, vp, C.c_double, vp, vp, C.c_double, vp, vp]
        lib.oracle_advec_dh_seed.restype = i32
        lib.oracle_advec_dh_seed.argtypes = [i32, vp, vp, vp, C.c_double, vp, vp]
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


class DhGrid:
    """The direct-hop grid of a 2-D advection mesh: box = {min x, y, z, max x, y, z} (z = 0),
    dims (X, Y, 1), spacing, and the map (x fastest), as the oracle builds it."""

    def __init__(self, box, dims, spacing, map_):
        self.box, self.dims, self.spacing, self.map = box, dims, spacing, map_
        self.inv = 1.0 / spacing


def dh_grid(c_pos_ll, spacing: float, expansion) -> tuple[np.ndarray, np.ndarray]:
    """BoundingBox(c_pos_ll, 2, expansion) and the CellMapper's box counts: (box[6], dims[3])."""
    ll = np.ascontiguousarray(c_pos_ll, dtype=np.float64)
    ex = np.ascontiguousarray(expansion, dtype=np.float64)
    box, dims = np.zeros(6), np.zeros(3, np.int64)
    if _lib().oracle_advec_dh_grid_init(len(ll), _p(ll), spacing, _p(ex), _p(box), _p(dims)) != 0:
        raise ValueError("grid too large")
    return box, dims


def dh_build(c_pos_ll, cell_width: float, extents, spacing: float, expansion) -> DhGrid:
    """The reference's structured map of the mesh, by its own search over all cells per query."""
    ll = np.ascontiguousarray(c_pos_ll, dtype=np.float64)
    box, dims = dh_grid(ll, spacing, expansion)
    ext = np.ascontiguousarray(extents, dtype=np.float64)
    m = np.zeros(int(dims[0] * dims[1]), np.int32)
    _lib().oracle_advec_dh_build(len(ll), _p(ll), cell_width, _p(ext), _p(box), spacing, _p(dims), _p(m))
    return DhGrid(box, dims, spacing, m)


def dh_seed(pos, p2c, g: DhGrid) -> int:
    """The global-move pre-pass in place (pos [n,2], p2c [n]); returns the particles removed."""
    return int(_lib().oracle_advec_dh_seed(len(p2c), _p(pos), _p(p2c), _p(g.box), g.inv, _p(g.dims), _p(g.map)))


def steps_dh(pos, vel, mdir, p2c, c2c, c_pos_ll, dt, extents, cell_width, n_steps, g: DhGrid,
             max_hops=1 << 20) -> tuple[int, int]:
    """steps() with every move starting from the direct-hop seed; returns (move calls of the
    last step, particles removed by the pre-pass)."""
    ext = np.ascontiguousarray(extents, dtype=np.float64)
    visits, removed = C.c_int64(0), C.c_int64(0)
    rc = _lib().oracle_advec_steps_dh(len(p2c), _p(pos), _p(vel), _p(mdir), _p(p2c), _p(c2c), _p(c_pos_ll), dt,
                                      _p(ext), cell_width, n_steps, max_hops, _p(g.map), _p(g.box), g.inv,
                                      _p(g.dims), C.byref(visits), C.byref(removed))
    if rc != 0:
        raise RuntimeError("oracle: a particle exceeded max_hops")
    return int(visits.value), int(removed.value)


def move(pos, mdir, p2c, c2c, c_pos_ll, extents, cell_width, g: DhGrid | None = None,
         max_hops=1 << 20) -> tuple[int, int]:
    """The move loop alone, in place (mdir, p2c), from the direct-hop seed when g is given;
    returns (move calls, particles removed by the pre-pass)."""
    ext = np.ascontiguousarray(extents, dtype=np.float64)
    visits, removed = C.c_int64(0), C.c_int64(0)
    args = (None, None, 0.0, None) if g is None else (_p(g.map), _p(g.box), g.inv, _p(g.dims))
    rc = _lib().oracle_advec_move_dh(len(p2c), _p(pos), _p(mdir), _p(p2c), _p(c2c), _p(c_pos_ll), _p(ext),
                                     cell_width, max_hops, *args, C.byref(visits), C.byref(removed))
    if rc != 0:
        raise RuntimeError("oracle: a particle exceeded max_hops")
    return int(visits.value), int(removed.value)


def steps_job(args) -> tuple:
    """One instance's n_steps in a worker process (args: pos, vel, mdir, p2c, c2c, c_pos_ll, dt,
    extents, cell_width, n_steps); returns (pos, mdir, p2c, move calls of the last step)."""
    pos, vel, mdir, p2c, c2c, c_pos_ll, dt, extents, cell_width, n_steps = args
    pos, mdir, p2c = pos.copy(), mdir.copy(), p2c.copy()
    v = steps(pos, vel, mdir, p2c, c2c, c_pos_ll, dt, extents, cell_width, n_steps)
    return pos, mdir, p2c, v


def run_reference(kind: str, nx, ny, cell_width, dt, pos, vel, mdir, p2c, c2c, c_pos_ll, n_steps,
                  threads: int | None = None, dh_spacing: float | None = None) -> dict:
    """Run oracle/_ref/advec_ref_{seq,omp}: n_steps of update_pos + move.  Returns per-step wall
    times and the final pos, mdir, p2c; with dh_spacing, the global move is on (the app's
    opp_init_direct_hop_cg with that grid spacing and an expansion of two cell widths in x and
    y) and the result also holds the reference's grid: dims, box and map."""
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
    hdr["magic"] = b"OPPBADV1" if dh_spacing is None else b"OPPBADV2"
    hdr["ints"] = [nx, ny, n, n_steps]
    hdr["dbl"] = [dt, cell_width]
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        with open(d / "case.bin", "wb") as f:
            f.write(hdr.tobytes())
            if dh_spacing is not None:
                f.write(np.array([1, 0], "<i4").tobytes() + np.array([dh_spacing], "<f8").tobytes())
            for a, t in ((c2c, "<i4"), (c_pos_ll, "<f8"), (pos, "<f8"), (vel, "<f8"), (mdir, "<i4"),
                         (p2c, "<i4")):
                f.write(np.ascontiguousarray(a, dtype=t).tobytes())
        (d / "params.txt").write_text(params_text("HoleFill_All", 10, 2.0, global_move=dh_spacing is not None))
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
    out = {"times": times, "pos": take("<f8", size * 2).reshape(size, 2),
           "mdir": take("<i4", size * 2).reshape(size, 2), "p2c": take("<i4", size)}
    if dh_spacing is not None:
        dims = take("<i8", 3)
        out["dims"], out["box"] = dims, take("<f8", 6)
        out["map"] = take("<i4", int(dims.prod()))
    return out
