"""The C++ drop-in path: a FemPIC main written against the opp_* API only
(op-pic_b200/apps/fempic/fempic_b200.cpp, linked with libopp_b200.so) runs on the GPU
and matches the oracle: identical sizes and removals per step, identical final particle
state (cells, positions, velocities, weights), node charges within 1e-12 relative."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from helpers import mesh
from oppb.fempic import injection_randoms
from oracle import oracle as O
from oracle import ref_runner as R

pytestmark = pytest.mark.gpu
APP = Path(__file__).resolve().parent.parent / "op-pic_b200" / "lib" / "fempic_b200"


@pytest.mark.parametrize("fill,period,steps", [("HoleFill_All", 10, 200), ("Sort_Periodic", 10, 200),
                                               ("Sort_Periodic", 5, 30)])
def test_fempic_app_matches_oracle(tmp_path, fill, period, steps):
    hm = mesh()
    inject = 2000
    dist = hm.inject_distribution(inject)
    tables = [injection_randoms(9, s, inject, 0.1) for s in range(steps)]
    R.write_case(tmp_path / "case.bin", hm, dist, steps, tables)
    (tmp_path / "params.txt").write_text(R.params_text(fill, period, 2.0))
    r = subprocess.run([str(APP), str(tmp_path / "params.txt"), str(tmp_path / "case.bin"), str(tmp_path / "out.bin")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = R.read_output(tmp_path / "out.bin", hm.n_nodes)

    o = O.OracleFemPIC(hm, dist, fill=fill, fill_period=period)
    for s in range(steps):
        out = o.step(tables[s])
        rec = got["records"][s]
        assert (int(rec["size"]), int(rec["removed"])) == (out["size"], out["removed"]), s
        n = o.size
        assert int(rec["h_p2c"]) == R.fnv1a(o.p2c[:n]), s
        assert int(rec["h_lc"]) == R.fnv1a(o.lc[:n]), s
    n = o.size
    assert got["size"] == n
    np.testing.assert_array_equal(got["p2c"], o.p2c[:n])
    np.testing.assert_array_equal(got["pos"].view(np.uint64), o.pos[:n].view(np.uint64))
    np.testing.assert_array_equal(got["vel"].view(np.uint64), o.vel[:n].view(np.uint64))
    np.testing.assert_array_equal(got["lc"].view(np.uint64), o.lc[:n].view(np.uint64))
    err = np.abs(got["node_charge"] - o.node_charge) / np.maximum(np.abs(o.node_charge), 1.0)
    assert err.max() <= 1e-12


def test_fempic_app_deterministic_deposit_repeats(tmp_path):
    """BOOL oppb_deterministic_deposit = true in the parameter file selects the integer
    fixed-point deposit: two runs give node charges identical bit for bit, particles equal to
    the oracle's and charges within 1e-12 of its sequential sums."""
    hm = mesh()
    inject, steps = 2000, 25
    dist = hm.inject_distribution(inject)
    tables = [injection_randoms(17, s, inject, 0.1) for s in range(steps)]
    R.write_case(tmp_path / "case.bin", hm, dist, steps, tables)
    (tmp_path / "params.txt").write_text(R.params_text("Sort_Periodic", 5, 2.0,
                                                       extra="BOOL oppb_deterministic_deposit = true\n"))
    outs = []
    for k in range(2):
        out = tmp_path / f"out{k}.bin"
        r = subprocess.run([str(APP), str(tmp_path / "params.txt"), str(tmp_path / "case.bin"), str(out)],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(R.read_output(out, hm.n_nodes))
    np.testing.assert_array_equal(outs[0]["node_charge"].view(np.uint64), outs[1]["node_charge"].view(np.uint64))
    o = O.OracleFemPIC(hm, dist, fill="Sort_Periodic", fill_period=5)
    for s in range(steps):
        o.step(tables[s])
    n = o.size
    np.testing.assert_array_equal(outs[0]["p2c"], o.p2c[:n])
    np.testing.assert_array_equal(outs[0]["lc"].view(np.uint64), o.lc[:n].view(np.uint64))
    err = np.abs(outs[0]["node_charge"] - o.node_charge) / np.maximum(np.abs(o.node_charge), 1.0)
    assert err.max() <= 1e-12


def test_fempic_app_global_move_matches_reference_golden(tmp_path):
    """The app with opp_global_move on (opp::BoundingBox + opp_init_direct_hop_cg, the
    reference app's set-up) against the reference seq backend's own global-move run
    (tests/golden/fempic_4x4x8_dh.npz): per-step sizes, removals and digests, final state."""
    from oppb.fempic import HostMesh

    z = np.load(Path(__file__).resolve().parent / "golden" / "fempic_4x4x8_dh.npz")
    hm = HostMesh(*[float(v) if i >= 3 else int(v) for i, v in enumerate(z["dims"])])
    steps, sp = int(z["steps"]), float(z["spacing"])
    R.write_case(tmp_path / "case.bin", hm, z["dist"], steps, list(z["tables"]), dt=float(z["dt"]),
                 dh=(sp, (4 * sp,) * 3))
    (tmp_path / "params.txt").write_text(R.params_text(str(z["fill"]), int(z["period"]), 2.0, global_move=True))
    r = subprocess.run([str(APP), str(tmp_path / "params.txt"), str(tmp_path / "case.bin"), str(tmp_path / "out.bin")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = R.read_output(tmp_path / "out.bin", hm.n_nodes)
    for s in range(steps):
        g, ref = got["records"][s], z["records"][s]
        assert (int(g["size"]), int(g["removed"])) == (int(ref["size"]), int(ref["removed"])), s
        assert int(g["h_p2c"]) == int(ref["h_p2c"]), s
        assert int(g["h_pos"]) == int(ref["h_pos"]), s
        assert int(g["h_lc"]) == int(ref["h_lc"]), s
    np.testing.assert_array_equal(got["p2c"], z["p2c"])
    np.testing.assert_array_equal(got["lc"].view(np.uint64), z["lc"].view(np.uint64))
    err = np.abs(got["node_charge"] - z["node_charge"]) / np.maximum(np.abs(z["node_charge"]), 1.0)
    assert err.max() <= 1e-12


def test_fempic_app_field_phase_matches_oracle(tmp_path):
    """The app with the reference main's field phase, through the opp_* API only:
    init_boundary_pot, FESolver (set-up, enrich_cell_shape_deriv, compute_phi),
    compute_node_charge_density, opp_reset_dat + compute_electric_field and the two OPP_MAX
    logging loops, with the reference's physical constants, against the oracle running the
    same phase (FemPIC's QE, EPS0, Kb; plasma_den 1e9, electron_temperature 1e6 K)."""
    from oppb.fempic import HostMesh
    from oracle import field as F

    hm = HostMesh(10, 10, 40, 1.0, 1.0, 4.0)
    hm_o = HostMesh(10, 10, 40, 1.0, 1.0, 4.0)  # the oracle rewrites its mesh's c_ef
    inject, steps, dt, wall, spwt = 2000, 10, 0.05, 1.0, 2e5
    n0, temp = 1e9, 1e6
    dist = hm.inject_distribution(inject)
    tables = [injection_randoms(31, s, inject, 0.1) for s in range(steps)]
    R.write_case(tmp_path / "case.bin", hm, dist, steps, tables, dt=dt, field=(wall, spwt))
    (tmp_path / "params.txt").write_text(R.params_text(
        "HoleFill_All", 10, 2.0, print_final=True,
        extra=f"REAL plasma_den = {n0}\nREAL electron_temperature = {temp}\n"))
    r = subprocess.run([str(APP), str(tmp_path / "params.txt"), str(tmp_path / "case.bin"), str(tmp_path / "out.bin")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "max_c_ef" in r.stdout + r.stderr and "did not converge" not in r.stdout + r.stderr
    got = R.read_output(tmp_path / "out.bin", hm.n_nodes)

    bnd = np.where(hm_o.n_type == 3, -1.0 * wall, 0.0)  # init_boundary_pot_kernel
    fs = F.FieldSystem(hm_o.n_pos, hm_o.n_type, bnd, hm_o.c2n)
    consts = F.FieldConsts(n0=n0, phi0=0.0, kte=8.617333262e-5 * temp, qe=1.602e-19, eps0=8.8541878e-12,
                           max_iter=10000)
    o = O.OracleFemPIC(hm_o, dist, dt=dt, field=(fs, consts, spwt, hm_o.n_vol))
    for s in range(steps):
        out = o.step(tables[s])
        rec = got["records"][s]
        assert (int(rec["size"]), int(rec["removed"])) == (out["size"], out["removed"]), s
    n = o.size
    np.testing.assert_array_equal(got["p2c"], o.p2c[:n])
    assert np.abs(got["pos"] - o.pos[:n]).max() <= 1e-9 * np.abs(o.pos[:n]).max()
    den = got["node_charge"]  # n_charge_den after compute_node_charge_density
    assert np.abs(den - o.node_charge).max() <= 1e-9 * np.abs(o.node_charge).max()
    assert np.abs(hm_o.c_ef - hm.c_ef).max() > 1e-6 * np.abs(hm.c_ef).max()  # the field phase changed the field


def test_fempic_app_shuffle_holds_the_oracles_particles(tmp_path):
    """opp_fill = Shuffle_Periodic through the drop-in runtime: the same sizes and removals as
    the oracle's sorted run every step, and at the end the same particles (the seq backend's
    shuffle sorts by cell; the GPU orders live particles by random keys)."""
    hm = mesh()
    inject, steps, period = 2000, 60, 4
    dist = hm.inject_distribution(inject)
    tables = [injection_randoms(13, s, inject, 0.1) for s in range(steps)]
    R.write_case(tmp_path / "case.bin", hm, dist, steps, tables)
    (tmp_path / "params.txt").write_text(R.params_text("Shuffle_Periodic", period, 2.0))
    r = subprocess.run([str(APP), str(tmp_path / "params.txt"), str(tmp_path / "case.bin"), str(tmp_path / "out.bin")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = R.read_output(tmp_path / "out.bin", hm.n_nodes)
    o = O.OracleFemPIC(hm, dist, fill="Sort_Periodic", fill_period=period)
    for s in range(steps):
        out = o.step(tables[s])
        rec = got["records"][s]
        assert (int(rec["size"]), int(rec["removed"])) == (out["size"], out["removed"]), s
    n = o.size

    def rows(p2c, pos, vel, lc):
        rec = np.concatenate([p2c.astype(np.int64)[:, None].view(np.uint64), pos.view(np.uint64),
                              vel.view(np.uint64), lc.view(np.uint64)], axis=1)
        return rec[np.lexsort(rec.T[::-1])]

    np.testing.assert_array_equal(rows(got["p2c"], got["pos"], got["vel"], got["lc"]),
                                  rows(o.p2c[:n], o.pos[:n], o.vel[:n], o.lc[:n]))
    assert np.any(np.diff(got["p2c"]) < 0)  # live particles not in cell order
    err = np.abs(got["node_charge"] - o.node_charge) / np.maximum(np.abs(o.node_charge), 1.0)
    assert err.max() <= 1e-12


def test_fempic_app_refuses_unknown_fill(tmp_path):
    """An opp_fill value that is no fill type aborts at opp_init instead of running on."""
    hm = mesh(4, 4, 8, 1.0, 1.0, 2.0)
    dist = hm.inject_distribution(100)
    R.write_case(tmp_path / "case.bin", hm, dist, 2, [injection_randoms(1, s, 100, 0.1) for s in range(2)])
    (tmp_path / "params.txt").write_text(R.params_text("Shuffle_Sometimes", 4, 2.0))
    r = subprocess.run([str(APP), str(tmp_path / "params.txt"), str(tmp_path / "case.bin"), str(tmp_path / "out.bin")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "fill" in (r.stdout + r.stderr)


REF_MAIN = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "fempic_opp_dropin"
LOG_LINE = re.compile(r"ts: (\d+)\s+np: (\d+) \((\d+) added, (\d+) removed\)\s+max c_ef: (\S+) max n_pot: (\S+)")


@pytest.mark.skipif(not REF_MAIN.exists(), reason="the reference's generated main was not built (oracle/Makefile)")
@pytest.mark.parametrize("fill,period,global_move", [("HoleFill_All", 10, False), ("Sort_Periodic", 5, False),
                                                     ("HoleFill_All", 10, True)])
def test_reference_generated_main_runs_on_the_dropin(tmp_path, fill, period, global_move):
    """The reference's own generated FemPIC main, apps_codegen/app_fempic_cg/fempic_opp.cpp,
    compiled unmodified against include/ and linked with libopp_b200.so (oracle/Makefile): its
    mesh from the app's text files through its own load_mesh(), its injection from its own
    init_inject_distributions and rand_file, the field phase every step (FESolver on the GPU),
    the physical constants of fempic_defs.h.  Its per-step log (particles, added, removed, max
    c_ef, max n_pot) against the oracle running the same step with the same field phase.  With
    opp_global_move on, the main's own BoundingBox and opp_init_direct_hop_cg build the grid (on
    the GPU here) and every move starts from it, as the oracle's global move does."""
    from oracle import field as F
    from oracle import mesh as OM

    # 0.08 per step along z: ions reach the far wall from step ~50; ~10 per inlet face per step
    dims, steps = (10, 10, 40, 1.0, 1.0, 4.0), 70
    n0, vion, temp, wall, spwt, dt = 1e9, 1e6, 1e6, 1.0, 4e4, 8e-8
    files = OM.write_box_files(dims, tmp_path)
    rand = np.random.default_rng(3).random((1000, 2))
    (tmp_path / "rand.dat").write_text("1000 2\n" + "".join(f"{float(a)!r} {float(b)!r}\n" for a, b in rand))
    (tmp_path / "params.txt").write_text(
        f"REAL plasma_den = {n0}\nREAL ion_velocity = {vion}\nREAL electron_temperature = {temp}\n"
        f"REAL wall_potential = {wall}\nREAL spwt = {spwt}\nINT charge_multiple = 1\nINT num_steps = {steps}\n"
        f"REAL dt = {dt}\nREAL grid_spacing = 0.1\nBOOL print_final = true\n"
        f"STRING global_mesh = {files['global_mesh']}\nSTRING inlet_mesh = {files['inlet_mesh']}\n"
        f"STRING wall_mesh = {files['wall_mesh']}\nSTRING rand_file = {tmp_path / 'rand.dat'}\n"
        f"STRING opp_fill = {fill}\nINT opp_fill_period = {period}\nREAL opp_allocation_multiple = 11\n"
        f"BOOL opp_global_move = {'true' if global_move else 'false'}\nBOOL opp_dh_data_generate = true\n"
        "BOOL opp_profile_all = false\n")
    r = subprocess.run([str(REF_MAIN), str(tmp_path / "params.txt")], capture_output=True, text=True, timeout=600,
                       cwd=tmp_path)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    log = [LOG_LINE.search(line) for line in r.stdout.splitlines()]
    log = [(int(m[1]), int(m[2]), int(m[3]), int(m[4]), float(m[5]), float(m[6])) for m in log if m]
    assert [x[0] for x in log] == list(range(steps))

    # The oracle: the loader's mesh (pinned by tests/test_mesh_ref_cpu.py), init_inject_distributions'
    # counts (plasma_den * ion_velocity * area * dt / spwt, truncated, per face), the rand_file's
    # pairs restarting at every face, no thermal velocity, charge / mass = QE / (2 AMU).
    qe, amu, kb, eps0 = 1.602e-19, 1.660538921e-27, 8.617333262e-5, 8.8541878e-12
    m = OM.box_mesh(*dims)
    per_face = [int(n0 * vion * a * dt / spwt + 0.0) for a in m.if_area]
    dist = np.cumsum(per_face).astype(np.int32)
    inject = int(dist[-1])
    start = np.concatenate([[0], dist[:-1]])
    face = np.searchsorted(dist, np.arange(inject), side="right")
    table = np.zeros((inject, 5))
    table[:, 0:2] = rand[np.arange(inject) - start[face]]
    bnd = np.where(m.n_type == OM.FIXED, -1.0 * wall, 0.0)  # init_boundary_pot_kernel
    fs = F.FieldSystem(m.n_pos, m.n_type, bnd, m.c2n)
    consts = F.FieldConsts(n0=n0, phi0=0.0, kte=kb * temp, qe=qe, eps0=eps0, max_iter=10000)
    dh = O.DirectHop(m.n_pos, 0.1, (0.4, 0.4, 0.4), mesh=m) if global_move else None  # grid_spacing, 4 x it
    o = O.OracleFemPIC(m, dist, ion_velocity=vion, qm=(1 * qe) / (2 * amu), dt=dt, fill=fill, fill_period=period,
                       field=(fs, consts, spwt, m.n_vol), dh=dh)
    removed = 0
    for s in range(steps):
        out = o.step(table)
        ts, np_, added, rem, max_cef, max_pot = log[s]
        assert (np_, added, rem) == (out["size"], inject, out["removed"]), s
        removed += rem
        assert abs(max_cef - max(0.0, float(m.c_ef.max()))) <= 1e-9 * max(1.0, abs(max_cef)), s
        assert abs(max_pot - float(np.abs(o.potential).max())) <= 1e-9 * max(1.0, abs(max_pot)), s
    assert removed > 0 and log[-1][1] > 50_000


ADV_SEQ = REF_MAIN.parent / "advec_opp_seq"
ADV_DROPIN = REF_MAIN.parent / "advec_opp_dropin"
ADV_LOG = re.compile(r"^Main\[\d+\]\[\d+\] - ts: .*$")


@pytest.mark.skipif(not (ADV_SEQ.exists() and ADV_DROPIN.exists()),
                    reason="the NESO-advection generated main was not built (oracle/Makefile)")
@pytest.mark.parametrize("global_move,nx,ny,ppc,steps", [(False, 128, 96, 50, 200), (True, 96, 64, 40, 120)])
def test_reference_advection_main_runs_on_the_dropin(tmp_path, global_move, nx, ny, ppc, steps):
    """The reference's generated NESO-advection main (apps_codegen/app_neso_advection_mdir_cg/
    advec_opp.cpp), unmodified, built twice by oracle/Makefile: on the reference's seq backend with
    its generated seq loops, and on include/ + libopp_b200.so.  Both with opp_exit wrapped to write
    every particle dat (oracle/dump_at_exit.cpp).  Same parameter file: the app's own init_mesh,
    its seeded init_particles, verify_particles every step, with and without the global move
    (direct-hop grid built by the seq backend's all-cell search there, on the GPU here).  The
    per-step log lines (errors, particle counts, hop bound) and the final particle dats (positions,
    velocities, move directions, cells, indices), with the cell dats, are equal byte for byte."""
    params = (f"INT num_steps = {steps}\nINT nx = {nx}\nINT ny = {ny}\nREAL dt = 0.5\nREAL cell_width = 0.5\n"
              f"INT npart_per_cell = {ppc}\nBOOL verify_particles = true\nREAL opp_allocation_multiple = 1.1\n"
              "INT opp_threads_per_block = 512\nBOOL opp_profile_all = false\n"
              f"BOOL opp_global_move = {'true' if global_move else 'false'}\nREAL grid_spacing = 0.5\n"
              "BOOL opp_dh_data_generate = true\nSTRING opp_fill = HoleFill_All\nINT opp_fill_period = 4\n")
    out = {}
    for name, exe in (("seq", ADV_SEQ), ("cuda", ADV_DROPIN)):
        d = tmp_path / name
        (d / "files").mkdir(parents=True)
        (d / "params.txt").write_text(params)
        r = subprocess.run([str(exe), "params.txt"], capture_output=True, text=True, timeout=600, cwd=d)
        assert r.returncode == 0, (name, r.stdout[-2000:], r.stderr[-2000:])
        log = [ln for ln in r.stdout.splitlines() if ADV_LOG.match(ln)]
        files = {p.name.replace(f"final_{name}_", ""): p.read_bytes() for p in (d / "files").iterdir()}
        out[name] = (log, files)
    log_seq, files_seq = out["seq"]
    log_gpu, files_gpu = out["cuda"]
    assert len(log_seq) == steps and all("errors: 0 |" in ln for ln in log_seq)
    assert f"Gbl parts: {nx * ny * ppc} " in log_seq[-1]
    assert log_gpu == log_seq
    assert sorted(files_gpu) == sorted(files_seq)
    assert {"p_index", "p_mesh_rel", "p_move_dir", "p_pos", "p_vel", "c_pos_ll"} <= set(files_seq)
    for k in files_seq:
        assert files_gpu[k] == files_seq[k], k


CAB_SEQ = REF_MAIN.parent / "cabana_opp_seq"
CAB_DROPIN = REF_MAIN.parent / "cabana_opp_dropin"
CAB_LOG = re.compile(r"ts: (\d+)\s+e_energy: \s*(\S+) b_energy: \s*(\S+) max_jx: (\S+) max_ex: (\S+) max_bx: (\S+)")


def read_dump(path: Path) -> np.ndarray:
    """A file of opp_print_dat_to_txtfile: the header, one row of values per element, the two
    marker lines."""
    lines = path.read_text().splitlines()
    size, dim = (int(v) for v in lines[0].split()[:2])
    rows = [ln.split() for ln in lines[1:1 + size]]
    assert all(len(r) == dim for r in rows) and lines[1 + size].startswith("import_exec_below")
    return np.array(rows, dtype=np.float64).reshape(size, dim)


@pytest.mark.skipif(not (CAB_SEQ.exists() and CAB_DROPIN.exists()),
                    reason="the CabanaPIC generated main was not built (oracle/Makefile)")
@pytest.mark.parametrize("nx,ny,nz,ppc,steps", [(8, 8, 24, 40, 25), (16, 16, 32, 60, 40)])
def test_reference_cabana_main_runs_on_the_dropin(tmp_path, nx, ny, nz, ppc, steps):
    """The reference's generated CabanaPIC main (apps_codegen/app_cabanapic_cg/cabana_opp.cpp),
    unmodified, built on the reference's seq backend and on include/ + libopp_b200.so
    (oracle/Makefile), opp_exit wrapped to write every dat (oracle/dump_at_exit.cpp): the app's own
    mesh, its two-stream particles, the whole step (field interpolation, move + current deposit,
    accumulation, the leapfrog B and E updates with their ghost copies) for `steps` steps.  The
    masks, indices and cells equal; the fields, accumulators and particles, and the per-step energy
    and maxima of the log and energy.csv, within 1e-9 of their largest values (B on E's scale):
    the current deposit adds FP64 atomics in a different order than the seq loop, and the energy
    is summed in a different order, so the two runs part at rounding level and the field
    feedback carries that forward."""
    params = (f"INT num_steps = {steps}\nREAL init_vel = 0.0866025403784439\nINT num_part_per_cell = {ppc}\n"
              f"INT nx = {nx}\nINT ny = {ny}\nINT nz = {nz}\nREAL c = 1.0\nREAL qsp = -1.0\nREAL me = 1.0\n"
              "REAL default_grid_len = 1.0\nREAL eps = 1.0\nSTRING part_enrich = two_stream\n"
              "BOOL print_energy = true\nSTRING cluster = block\nREAL opp_allocation_multiple = 1.1\n"
              "INT opp_threads_per_block = 256\nBOOL opp_profile_all = false\nBOOL print_final = true\n"
              "STRING opp_fill = HoleFill_All\nINT opp_fill_period = 4\nBOOL opp_global_move = false\n"
              "INT domain_expansion = 1\nREAL velX_mult_const = 1\nREAL velY_mult_const = 0.00\n"
              "REAL velZ_mult_const = 0.00\n")
    out = {}
    for name, exe in (("seq", CAB_SEQ), ("cuda", CAB_DROPIN)):
        d = tmp_path / name
        (d / "files").mkdir(parents=True)
        (d / "params.txt").write_text(params)
        r = subprocess.run([str(exe), "params.txt"], capture_output=True, text=True, timeout=600, cwd=d)
        assert r.returncode == 0, (name, r.stdout[-2000:], r.stderr[-2000:])
        log = [m.groups() for m in map(CAB_LOG.search, r.stdout.splitlines()) if m]
        energy = np.loadtxt(d / "energy.csv", delimiter=",", skiprows=1)
        dats = {p.name.replace(f"final_{name}_", ""): read_dump(p) for p in (d / "files").iterdir()}
        out[name] = (np.array(log, dtype=np.float64), energy, dats)
    log_s, en_s, dats_s = out["seq"]
    log_g, en_g, dats_g = out["cuda"]
    assert log_s.shape == log_g.shape == (steps, 6) and en_s.shape == en_g.shape == (steps, 3)
    np.testing.assert_array_equal(log_g[:, 0], np.arange(steps))
    assert en_s[-1, 1] > 10 * en_s[0, 1] > 0  # the electric energy grows: the run is not trivial
    assert sorted(dats_g) == sorted(dats_s)
    assert {"p_pos", "p_vel", "p_streak_mid", "p_weight", "p2c_map", "c_e", "c_b", "c_j", "c_acc"} <= set(dats_s)
    # E and B share their units (c = 1): B, which stays at rounding level in this workload, is
    # compared on E's scale, and so is the magnetic energy on the electric energy's.
    e_scale = np.abs(dats_s["c_e"]).max()
    scale = {"c_b": e_scale, "c_e": e_scale, "c_interp": e_scale}
    err = {}
    for k in dats_s:
        a, b = dats_g[k], dats_s[k]
        assert a.shape == b.shape, k
        if k.startswith("c_mask") or k in ("c_index", "c_colors", "p2c_map"):
            np.testing.assert_array_equal(a, b, err_msg=k)
        else:
            err[k] = np.abs(a - b).max() / max(scale.get(k, np.abs(b).max()), 1e-300)
    e_energy = np.abs(en_s[:, 1]).max()
    err["e_energy"] = np.abs(en_g[:, 1] - en_s[:, 1]).max() / e_energy
    err["b_energy"] = np.abs(en_g[:, 2] - en_s[:, 2]).max() / e_energy
    # the logged maxima of jx, ex, bx, printed with 10, 10 and 16 decimals
    err["max_jx"] = (np.abs(log_g[:, 3] - log_s[:, 3]).max() - 1e-10) / np.abs(log_s[:, 3]).max()
    err["max_ex"] = (np.abs(log_g[:, 4] - log_s[:, 4]).max() - 1e-10) / e_scale
    err["max_bx"] = (np.abs(log_g[:, 5] - log_s[:, 5]).max() - 1e-16) / e_scale
    assert max(err.values()) <= 1e-9, err
