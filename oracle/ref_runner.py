"""TEST INFRASTRUCTURE ONLY — runs the compiled OP-PIC reference (oracle/_ref, built by
oracle/Makefile from the reference sources) on a FemPIC case and reads back its per-step
records (sizes, FNV-1a digests of the particle dats and node charges, wall times).

Box cases (run_box, box_mesh) take the mesh from the reference app's own loader: the harness
writes the box as the app's text mesh files and loads them with load_mesh()
(apps_codegen/app_fempic_cg/fempic_misc_mesh_loader.h), so nothing of the library under test
is involved.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parent / "_ref"
BINARIES = {"seq_stable": "fempic_ref_seq_stable", "seq": "fempic_ref_seq", "omp": "fempic_ref_omp"}
STEP_DTYPE = np.dtype([("step", "<i4"), ("size_before_move", "<i4"), ("removed", "<i4"), ("size", "<i4"),
                       ("h_p2c", "<u8"), ("h_pos", "<u8"), ("h_vel", "<u8"), ("h_lc", "<u8"), ("h_charge", "<u8"),
                       ("t_inject", "<f8"), ("t_push", "<f8"), ("t_move", "<f8"), ("t_deposit", "<f8")])


def available(kind: str = "seq_stable") -> bool:
    return (REF_DIR / BINARIES[kind]).exists()


def fnv1a(a: np.ndarray) -> int:
    from oracle.oracle import load

    lib = load()
    lib.oracle_fnv1a.restype = C.c_uint64
    lib.oracle_fnv1a.argtypes = [C.c_void_p, C.c_int64]
    a = np.ascontiguousarray(a)
    return int(lib.oracle_fnv1a(a.ctypes.data, a.nbytes))


def write_case(path: Path, mesh, dist: np.ndarray, steps: int, tables: list[np.ndarray], dt: float = 0.01,
               qm: float = 1.0, ion_velocity: float = 1.0, sigma: float = 0.1, record_state: bool = True,
               dh: tuple | None = None, field: tuple | None = None) -> None:
    """dh = (grid_spacing, expansion[3]): a global-move case; the node positions follow.
    field = (wall_potential, spwt): a block tagged OPPBFLD1 at the end with the node types,
    positions and volumes, for the library's FemPIC app with its field phase (the reference
    harness does not read it)."""
    inject = int(dist[-1])
    hdr = np.zeros(1, dtype=[("magic", "S8"), ("ints", "<i4", 8), ("dbl", "<f8", 4)])
    hdr["magic"] = b"OPPBCAS1"
    hdr["ints"] = [mesh.n_nodes, mesh.n_cells, mesh.n_ifaces, inject, steps, len(tables), int(record_state),
                   int(dh is not None)]
    hdr["dbl"] = [dt, qm, ion_velocity, sigma]
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        for a, dt_ in ((mesh.c2n, "<i4"), (mesh.c2c, "<i4"), (mesh.c_det, "<f8"), (mesh.c_vol, "<f8"),
                       (mesh.c_ef, "<f8"), (mesh.if2c, "<i4"), (mesh.if_u, "<f8"), (mesh.if_v, "<f8"),
                       (mesh.if_norm, "<f8"), (mesh.if_n_pos, "<f8"), (dist, "<i4")):
            f.write(np.ascontiguousarray(a, dtype=dt_).tobytes())
        for t in tables:
            assert t.shape == (inject, 5)
            f.write(np.ascontiguousarray(t, dtype="<f8").tobytes())
        if dh is not None:
            spacing, expansion = dh
            f.write(np.array([spacing, *expansion], "<f8").tobytes())
            f.write(np.ascontiguousarray(mesh.n_pos, dtype="<f8").tobytes())
        if field is not None:
            f.write(b"OPPBFLD1")
            f.write(np.ascontiguousarray(mesh.n_type, dtype="<i4").tobytes())
            f.write(np.ascontiguousarray(mesh.n_pos, dtype="<f8").tobytes())
            f.write(np.ascontiguousarray(mesh.n_vol, dtype="<f8").tobytes())
            f.write(np.array(field, "<f8").tobytes())


def params_text(fill: str, period: int, alloc_mult: float, global_move: bool = False, print_final: bool = False,
                extra: str = "") -> str:
    """The opp_* parameter file of a run; extra: more `TYPE key = value` lines."""
    gm = "true" if global_move else "false"
    pf = "true" if print_final else "false"
    return (f"STRING opp_fill = {fill}\nINT opp_fill_period = {period}\n"
            f"REAL opp_allocation_multiple = {alloc_mult}\nBOOL opp_profile_all = false\n"
            f"BOOL opp_global_move = {gm}\nBOOL opp_dh_data_generate = {gm}\n"
            f"INT opp_threads_per_block = 256\nBOOL print_final = {pf}\n" + extra)


BOX_DTYPE = np.dtype([("magic", "S8"), ("ints", "<i4", 8), ("dbl", "<f8", 9)])


def write_box_case(path: Path, dims, inject: int = 0, steps: int = 0, dt: float = 0.01, qm: float = 1.0,
                   ion_velocity: float = 1.0, sigma: float = 0.1, phi_inlet: float = 1.0, phi_fixed: float = 0.0,
                   record_state: bool = False, mesh_only: bool = False, seed: int = 0) -> None:
    """dims = (nx, ny, nz, lx, ly, lz): the box the harness writes and loads."""
    nx, ny, nz, lx, ly, lz = dims
    hdr = np.zeros(1, dtype=BOX_DTYPE)
    hdr["magic"] = b"OPPBBOX1"
    hdr["ints"] = [nx, ny, nz, inject, steps, int(record_state), int(mesh_only), seed]
    hdr["dbl"] = [lx, ly, lz, dt, qm, ion_velocity, sigma, phi_inlet, phi_fixed]
    Path(path).write_bytes(hdr.tobytes())


def mesh_params(d: Path) -> str:
    """The app's mesh-file parameters (apps_codegen/app_fempic_cg/configs/coarse.param) for files in d."""
    return (f"STRING global_mesh = {d / 'mesh.dat'}\nSTRING inlet_mesh = {d / 'inlet.dat'}\n"
            f"STRING wall_mesh = {d / 'wall.dat'}\n")


def box_mesh(dims, kind: str = "seq") -> dict:
    """The mesh arrays load_mesh() gives for the box dims = (nx, ny, nz, lx, ly, lz), in the
    app's host layout: n_pos, n_vol, n_type, c2n, c2c, c_det, c_vol, c_centroid, if2c, if2n,
    if_u, if_v, if_norm, if_area, if_n_pos."""
    exe = REF_DIR / BINARIES[kind]
    if not exe.exists():
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        write_box_case(d / "case.bin", dims, mesh_only=True)
        (d / "params.txt").write_text(params_text("HoleFill_All", 10, 2.0, extra=mesh_params(d)))
        r = subprocess.run([str(exe), str(d / "params.txt"), str(d / "case.bin"), str(d / "out.bin")],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{exe.name} failed ({r.returncode}): {r.stderr[-2000:]}")
        raw = (d / "out.bin").read_bytes()
    nn, nc, nf = (int(v) for v in np.frombuffer(raw[:12], "<i4"))
    off = 12
    out = {"n_nodes": nn, "n_cells": nc, "n_ifaces": nf}
    for name, dt, shape in (("n_pos", "<f8", (nn, 3)), ("n_vol", "<f8", (nn,)), ("n_type", "<i4", (nn,)),
                            ("c2n", "<i4", (nc, 4)), ("c2c", "<i4", (nc, 4)), ("c_det", "<f8", (nc, 16)),
                            ("c_vol", "<f8", (nc,)), ("c_centroid", "<f8", (nc, 3)), ("if2c", "<i4", (nf,)),
                            ("if2n", "<i4", (nf, 3)), ("if_u", "<f8", (nf, 3)), ("if_v", "<f8", (nf, 3)),
                            ("if_norm", "<f8", (nf, 3)), ("if_area", "<f8", (nf,)), ("if_n_pos", "<f8", (nf, 9))):
        n = int(np.prod(shape)) * np.dtype(dt).itemsize
        out[name] = np.frombuffer(raw[off:off + n], dt).reshape(shape).copy()
        off += n
    return out


def run_box(kind: str, dims, inject: int, steps: int, fill: str = "HoleFill_All", period: int = 10,
            alloc_mult: float = 2.0, threads: int | None = None, record_state: bool = False, seed: int = 0,
            **kw) -> dict:
    """The step loop on the box mesh loaded by the app's loader (the workload's injection
    distribution, the exact static field of its Laplace problem, the harness's own seeded
    randoms).  kw: dt, qm, ion_velocity, sigma, phi_inlet, phi_fixed."""
    exe = REF_DIR / BINARIES[kind]
    if not exe.exists():
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        write_box_case(d / "case.bin", dims, inject=inject, steps=steps, record_state=record_state, seed=seed, **kw)
        (d / "params.txt").write_text(params_text(fill, period, alloc_mult, extra=mesh_params(d)))
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        r = subprocess.run([str(exe), str(d / "params.txt"), str(d / "case.bin"), str(d / "out.bin")],
                           stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"{exe.name} failed ({r.returncode}): {r.stderr[-2000:]}")
        nn = int(np.prod([dims[0] + 1, dims[1] + 1, dims[2] + 1]))
        return read_output(d / "out.bin", nn, record_state)


def run(kind: str, mesh, dist, steps: int, tables, fill: str = "HoleFill_All", period: int = 10,
        alloc_mult: float = 2.0, record_state: bool = True, threads: int | None = None, **kw) -> dict:
    exe = REF_DIR / BINARIES[kind]
    if not exe.exists():
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        write_case(d / "case.bin", mesh, dist, steps, tables, record_state=record_state, **kw)
        (d / "params.txt").write_text(params_text(fill, period, alloc_mult, global_move=kw.get("dh") is not None))
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        r = subprocess.run([str(exe), str(d / "params.txt"), str(d / "case.bin"), str(d / "out.bin")],
                           capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"{exe.name} failed ({r.returncode}): {r.stderr[-2000:]}")
        return read_output(d / "out.bin", mesh.n_nodes, record_state, direct_hop=kw.get("dh") is not None)


def read_output(path: Path, n_nodes: int, record_state: bool = True, direct_hop: bool = False) -> dict:
    """Per-step records and final state written by the harness (and by the library's
    FemPIC app, which uses the same layout)."""
    raw = Path(path).read_bytes()
    nrec = int(np.frombuffer(raw[:4], "<i4")[0])
    off = 4
    recs = np.frombuffer(raw[off:off + nrec * STEP_DTYPE.itemsize], STEP_DTYPE).copy()
    off += nrec * STEP_DTYPE.itemsize
    fin = int(np.frombuffer(raw[off:off + 4], "<i4")[0])
    off += 4
    out = {"records": recs, "size": fin}
    if record_state:
        def take(dt, n):
            nonlocal off
            a = np.frombuffer(raw[off:off + n * np.dtype(dt).itemsize], dt).copy()
            off += n * np.dtype(dt).itemsize
            return a
        out["p2c"] = take("<i4", fin)
        out["pos"] = take("<f8", fin * 3).reshape(fin, 3)
        out["vel"] = take("<f8", fin * 3).reshape(fin, 3)
        out["lc"] = take("<f8", fin * 4).reshape(fin, 4)
        out["node_charge"] = take("<f8", n_nodes)
    if direct_hop:  # the reference's structured grid: box counts, bounds, map
        out["dh_dims"] = np.frombuffer(raw[off:off + 24], "<i8").copy()
        off += 24
        out["dh_box"] = np.frombuffer(raw[off:off + 48], "<f8").copy()
        off += 48
        n = int(np.prod(out["dh_dims"]))
        out["dh_map"] = np.frombuffer(raw[off:off + 4 * n], "<i4").copy()
    return out
