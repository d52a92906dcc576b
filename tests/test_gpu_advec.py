"""NESO-advection kernels through the C ABI: a batch of independent instances of different
meshes, particle counts and constants, advanced by one persistent launch per step, against the
oracle run on every instance alone; positions, move directions, cells and move-call counts
bit-exact.  Also the reference's own outputs (golden fixture), the separate update_pos / move
loops, CUDA-graph replay, and the error paths."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oppb import _lib as L
from oppb.advec import AdvecBatchDevice, AdvecMesh, particles
from oracle import advec as OA

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
GOLDEN = Path(__file__).resolve().parent / "golden" / "advec_13x9.npz"

# (nx, ny, cell_width, dt, ppc, v_sd): extents >= 1 on both axes (the reference's wrap needs it)
INSTANCES = [(13, 9, 0.7, 0.35, 30, 2.0), (40, 17, 1.0, 0.5, 7, 0.6), (7, 33, 0.3, 0.2, 11, 1.5),
             (64, 64, 1.0, 0.5, 50, 0.5), (4, 4, 1.0, 0.8, 3, 4.0)]


def _build(specs, seed0=0, grid=True):
    meshes = [AdvecMesh(nx, ny, cw) for nx, ny, cw, _, _, _ in specs]
    host = [particles(m, ppc, v_sd, seed0 + k) for k, (m, (_, _, _, _, ppc, v_sd)) in enumerate(zip(meshes, specs))]
    dev = AdvecBatchDevice(meshes, [len(h[3]) for h in host], [s[3] for s in specs], DEV, grid=grid)
    for k, h in enumerate(host):
        dev.set_instance(k, *h)
    return meshes, host, dev


def _oracle(meshes, host, specs, steps):
    out, visits = [], 0
    for m, (pos, vel, mdir, p2c), s in zip(meshes, host, specs):
        pos, mdir, p2c = pos.copy(), mdir.copy(), p2c.copy()
        for _ in range(steps):
            visits += OA.steps(pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, s[3], m.extents, m.cell_width, 1)
        out.append({"pos": pos, "mdir": mdir, "p2c": p2c})
    return out, visits


def _assert_same(dev, ref):
    for k, r in enumerate(ref):
        got = dev.host_instance(k)
        np.testing.assert_array_equal(got["pos"].view(np.uint64), r["pos"].view(np.uint64), err_msg=f"pos {k}")
        np.testing.assert_array_equal(got["mdir"], r["mdir"], err_msg=f"mdir {k}")
        np.testing.assert_array_equal(got["p2c"], r["p2c"], err_msg=f"p2c {k}")


@pytest.mark.parametrize("grid", [True, False], ids=["grid", "records"])
def test_batch_step_matches_oracle_per_instance(grid):
    """Cells verified as the periodic grid (corners and neighbours computed) and read from
    their records: the same results, the oracle's."""
    steps = 6
    meshes, host, dev = _build(INSTANCES, grid=grid)
    assert dev.grid_nx == ([m.nx for m in meshes] if grid else [0] * len(meshes))
    dev.zero_status()
    for _ in range(steps):
        dev.step()
    torch.cuda.synchronize()
    st = dev.status_host()
    ref, visits = _oracle(meshes, host, INSTANCES, steps)
    assert st.error == 0 and int(st.total_visits) == visits
    _assert_same(dev, ref)


def test_matches_reference_golden():
    z = np.load(GOLDEN)
    m = AdvecMesh(int(z["nx"]), int(z["ny"]), float(z["cell_width"]))
    dev = AdvecBatchDevice([m], [len(z["p2c"])], [float(z["dt"])], DEV)
    dev.set_instance(0, z["pos"], z["vel"], z["mdir"], z["p2c"])
    for _ in range(int(z["steps"])):
        dev.step()
    torch.cuda.synchronize()
    got = dev.host_instance(0)
    np.testing.assert_array_equal(got["pos"].view(np.uint64), z["ref_pos"].view(np.uint64))
    np.testing.assert_array_equal(got["mdir"], z["ref_mdir"])
    np.testing.assert_array_equal(got["p2c"], z["ref_p2c"])


def test_separate_loops_equal_fused_step():
    meshes, host, dev_a = _build(INSTANCES, seed0=20)
    _, _, dev_b = _build(INSTANCES, seed0=20)
    for _ in range(4):
        dev_a.step()
        dev_b.update_pos()
        dev_b.move()
    torch.cuda.synchronize()
    for k in range(len(INSTANCES)):
        a, b = dev_a.host_instance(k), dev_b.host_instance(k)
        for name in ("pos", "mdir", "p2c"):
            np.testing.assert_array_equal(a[name], b[name], err_msg=f"{name} {k}")
    assert int(dev_a.status_host().total_visits) == int(dev_b.status_host().total_visits)


def test_cuda_graph_replay_equals_launches():
    meshes, host, dev_a = _build(INSTANCES, seed0=40)
    _, _, dev_b = _build(INSTANCES, seed0=40)
    dev_a.zero_status()
    dev_b.zero_status()
    dev_a.step()  # sizes the persistent grid outside the capture
    dev_b.step()
    g = dev_b.capture(3)
    for _ in range(6):
        dev_a.step()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for k in range(len(INSTANCES)):
        a, b = dev_a.host_instance(k), dev_b.host_instance(k)
        for name in ("pos", "mdir", "p2c"):
            np.testing.assert_array_equal(a[name], b[name], err_msg=f"{name} {k}")
    assert int(dev_a.status_host().total_visits) == int(dev_b.status_host().total_visits)


def test_errors_reported():
    m = AdvecMesh(6, 6, 1.0)
    pos, vel, mdir, p2c = particles(m, 4, 0.5, 1)
    p2c[9] = 1000
    dev = AdvecBatchDevice([m], [len(p2c)], [0.5], DEV)
    dev.set_instance(0, pos, vel, mdir, p2c)
    dev.zero_status()
    dev.step()
    st = dev.status_host()
    assert st.error == L.OPPB_ERR_CELL_RANGE and st.error_index == 9
    # extents below 1 break the reference's wrap: the walk around the ring ends at the hop bound
    m2 = AdvecMesh(2, 2, 0.25)
    pos, vel, mdir, p2c = particles(m2, 2, 0.0, 2)
    vel[0] = (-40.0, 0.0)
    dev2 = AdvecBatchDevice([m2], [len(p2c)], [0.1], DEV)
    dev2.set_instance(0, pos, vel, mdir, p2c)
    dev2.zero_status()
    dev2.step(max_hops=64)
    st = dev2.status_host()
    assert st.error == L.OPPB_ERR_HOP_LIMIT and st.error_index == 0


def test_verify_kernel_invariant_on_a_large_batch():
    """The reference's verify_kernel (apps/app_neso_advection/kernels.h:115-151) after many steps
    of a batch of larger instances: every particle's position lies in the closed box
    [ix w, ix w + w] x [iy w, iy w + w] of its cell (ix, iy) = (cell mod nx, cell div nx), so the
    incorrect count is 0."""
    specs = [(128, 96, 1.0, 0.5, 60, 0.5), (200, 64, 0.25, 0.1, 25, 1.0), (33, 257, 0.7, 0.3, 40, 0.8),
             (256, 256, 1.0, 0.5, 20, 0.5)]
    meshes, _, dev = _build(specs, seed0=40)
    dev.zero_status()
    for _ in range(40):
        dev.step()
    torch.cuda.synchronize()
    assert dev.status_host().error == 0
    for k, m in enumerate(meshes):
        got = dev.host_instance(k)
        ix, iy = got["p2c"] % m.nx, got["p2c"] // m.nx
        w = m.cell_width
        llx, lly = ix * w, iy * w  # the reference's boundary_ll, in FP64
        x, y = got["pos"][:, 0], got["pos"][:, 1]
        incorrect = (ix < 0) | (iy < 0) | (x < llx) | (x > llx + w) | (y < lly) | (y > lly + w)
        assert int(incorrect.sum()) == 0, (k, int(incorrect.sum()))


def test_ensemble_of_64_over_500_steps_under_graph_matches_oracle():
    """Config 5 at its own scale and length: 64 instances with sides drawn from U{64..512} (the
    benchmark's seeded draw), |v dt| <= 0.5 cell, 500 steps advanced as 50 replays of a 10-step
    CUDA graph of the persistent launch; positions, move directions and cells of every
    instance bit-exact against the oracle run on each instance alone (worker processes).
    Particles per cell are drawn from U{1..3} instead of U{10..200}, so that the oracle's
    ~6e9 particle-steps finish in about a minute; the kernels, the in-order work counter and
    the graph see the same 64 uneven meshes."""
    import multiprocessing as mp
    import os

    rng = np.random.default_rng(5)
    sides = rng.integers(64, 513, 64)
    ppcs = rng.integers(1, 4, 64)
    specs = [(int(sd), int(sd), 1.0, 0.5, int(pc), 0.5) for sd, pc in zip(sides, ppcs)]
    meshes = [AdvecMesh(nx, ny, cw) for nx, ny, cw, _, _, _ in specs]
    host = [particles(m, s[4], s[5], 5000 + k, v_clip=1.0) for k, (m, s) in enumerate(zip(meshes, specs))]
    steps = 500
    jobs = [(h[0], h[1], h[2], h[3], m.c2c, m.c_pos_ll, s[3], np.array(m.extents, np.float64), m.cell_width, steps)
            for m, h, s in zip(meshes, host, specs)]
    ctx = mp.get_context("spawn")  # workers import only the oracle
    pool = ctx.Pool(max(1, min(len(jobs), len(os.sched_getaffinity(0)) - 1)))
    pending = pool.map_async(OA.steps_job, jobs, chunksize=1)
    dev = AdvecBatchDevice(meshes, [len(h[3]) for h in host], [s[3] for s in specs], DEV)
    for k, h in enumerate(host):
        dev.set_instance(k, *h)
    dev.zero_status()
    dev.step()  # sizes the persistent grid outside the capture
    g = dev.capture(10)
    for _ in range((steps - 1) // 10):
        g.replay()
    for _ in range((steps - 1) % 10):
        dev.step()
    torch.cuda.synchronize()
    assert dev.status_host().error == 0
    ref = pending.get(timeout=1800)
    pool.close()
    pool.join()
    assert sum(len(h[3]) for h in host) > 5_000_000
    _assert_same(dev, [{"pos": r[0], "mdir": r[1], "p2c": r[2]} for r in ref])


# ------------------------------------------------------------------ direct hop (global move)

GOLDEN_DH = Path(__file__).resolve().parent / "golden" / "advec_dh_9x8.npz"
# (nx, ny, cell_width, grid spacing): spacings that align with the cells, straddle their
# edges, or are coarser than a cell
DH_MESHES = [(9, 8, 1.0, 0.7), (13, 9, 0.5, 0.5), (7, 11, 1.0, 0.3), (10, 6, 0.25, 0.4), (5, 19, 0.8, 1.9),
             (64, 48, 1.0, 0.45)]


def test_dh_maps_match_oracle():
    """oppb_dh_build_quad (the cells binned into the grid boxes, one query thread per box)
    gives the oracle's map (the reference's search over all cells per query), and the grid's
    counts and bounds are the oracle's, for every instance of a batch."""
    meshes = [AdvecMesh(nx, ny, cw) for nx, ny, cw, _ in DH_MESHES]
    for m, (_, _, cw, gs) in zip(meshes, DH_MESHES):
        dev = AdvecBatchDevice([m], [1], [0.5], DEV)
        dev.enable_direct_hop(gs)
        g, gmap = dev.dh_grids[0]
        ref = OA.dh_build(m.c_pos_ll, cw, m.extents, gs, (2 * cw, 2 * cw, 0.0))
        assert list(g.dims) == list(ref.dims)
        np.testing.assert_array_equal(np.array(list(g.min) + list(g.max)).view(np.uint64), ref.box.view(np.uint64))
        np.testing.assert_array_equal(gmap.cpu().numpy(), ref.map, err_msg=str((m.nx, m.ny, cw, gs)))


def test_dh_matches_reference_golden():
    """The global move on, as the reference ran it (golden fixture): map, then 7 steps with
    particles on cell edges that the seed moves to the neighbouring cell."""
    z = np.load(GOLDEN_DH)
    cw = float(z["cell_width"])
    m = AdvecMesh(int(z["nx"]), int(z["ny"]), cw)
    dev = AdvecBatchDevice([m], [len(z["p2c"])], [float(z["dt"])], DEV)
    dev.set_instance(0, z["pos"], z["vel"], z["mdir"], z["p2c"])
    dev.enable_direct_hop(float(z["grid_spacing"]))
    np.testing.assert_array_equal(dev.dh_grids[0][1].cpu().numpy(), z["ref_map"])
    dev.zero_status()
    for _ in range(int(z["steps"])):
        dev.step()
    torch.cuda.synchronize()
    got = dev.host_instance(0)
    np.testing.assert_array_equal(got["pos"].view(np.uint64), z["ref_pos"].view(np.uint64))
    np.testing.assert_array_equal(got["mdir"], z["ref_mdir"])
    np.testing.assert_array_equal(got["p2c"], z["ref_p2c"])
    assert dev.status_host().remove_count == 0


@pytest.mark.parametrize("grid", [True, False], ids=["grid", "records"])
def test_dh_batch_steps_match_oracle_and_graph(grid):
    """A batch of the meshes above with edge particles: 12 steps with the seed, as launches and
    as replays of a 4-step CUDA graph, against the oracle per instance (positions, directions,
    cells, move calls)."""
    from helpers import advec_edge_particles

    meshes = [AdvecMesh(nx, ny, cw) for nx, ny, cw, _ in DH_MESHES]
    host = [advec_edge_particles(m, 9, 0.7, 300 + k) for k, m in enumerate(meshes)]
    dts = [0.45] * len(meshes)
    devs = []
    for _ in range(2):
        d = AdvecBatchDevice(meshes, [len(h[3]) for h in host], dts, DEV, grid=grid)
        for k, h in enumerate(host):
            d.set_instance(k, *h)
        devs.append(d)
    for d in devs:  # every instance with its own spacing
        d.enable_direct_hop([gs for _, _, _, gs in DH_MESHES])
    steps = 12
    a, b = devs
    a.zero_status()
    b.zero_status()
    for _ in range(steps):
        a.step()
    b.step()
    g = b.capture(4)
    for _ in range((steps - 1) // 4):
        g.replay()
    for _ in range((steps - 1) % 4):
        b.step()
    torch.cuda.synchronize()
    ref, visits = [], 0
    for m, h, (_, _, cw, gs), dt in zip(meshes, host, DH_MESHES, dts):
        pos, vel, mdir, p2c = (x.copy() for x in h)
        grid = OA.dh_build(m.c_pos_ll, cw, m.extents, gs, (2 * cw, 2 * cw, 0.0))
        for _ in range(steps):
            v, r = OA.steps_dh(pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, dt, m.extents, cw, 1, grid)
            visits += v
            assert r == 0
        ref.append({"pos": pos, "mdir": mdir, "p2c": p2c})
    sa, sb = a.status_host(), b.status_host()
    assert sa.error == 0 and int(sa.total_visits) == visits and sa.remove_count == 0
    assert int(sb.total_visits) == visits
    _assert_same(a, ref)
    _assert_same(b, ref)


def test_dh_move_only_removes_outside_the_grid():
    """oppb_advec_move with the seed: positions past the grid on either axis, or in a box
    without a cell, are removed (p2c = REMOVED, counted), particles already removed are
    skipped, the others walk from the seed as the oracle's move loop does."""
    m = AdvecMesh(12, 10, 1.0)
    pos, vel, mdir, p2c = particles(m, 6, 0.0, 8)
    n = len(p2c)
    rng = np.random.default_rng(3)
    pos += rng.normal(0.0, 1.5, pos.shape)  # away from their cells (multi-hop walks)
    pos[:, 0] = np.clip(pos[:, 0], 0.0, 11.999)
    pos[:, 1] = np.clip(pos[:, 1], 0.0, 9.999)
    pos[0] = (1e9, 3.0)    # past the grid in x
    pos[1] = (3.0, 1e9)    # past the grid in y
    pos[2] = (-1.7, 3.0)   # inside the grid, in a box left of the mesh: no cell
    pos[3] = (-1e9, -1e9)  # truncates to box (0, 0): no cell
    p2c[4] = 2147483647    # already removed: skipped
    dev = AdvecBatchDevice([m], [n], [0.5], DEV)
    dev.set_instance(0, pos, vel, mdir, p2c)
    dev.enable_direct_hop(0.6)
    dev.zero_status()
    dev.move()
    torch.cuda.synchronize()
    st = dev.status_host()
    g = OA.dh_build(m.c_pos_ll, 1.0, m.extents, 0.6, (2.0, 2.0, 0.0))
    P, M, C2 = pos.copy(), mdir.copy(), p2c.copy()
    visits, removed = OA.move(P, M, C2, m.c2c, m.c_pos_ll, m.extents, 1.0, g)
    got = dev.host_instance(0)
    assert st.error == 0 and st.remove_count == removed == 4
    assert int(st.total_visits) == visits
    np.testing.assert_array_equal(got["p2c"], C2)
    np.testing.assert_array_equal(got["mdir"], M)
    assert list(np.flatnonzero(C2 == 2147483647)) == [0, 1, 2, 3, 4]


def test_dh_disabled_walks_from_p2c_again():
    m = AdvecMesh(9, 8, 1.0)
    from helpers import advec_edge_particles

    pos, vel, mdir, p2c = advec_edge_particles(m, 10, 0.5, 11)
    dev = AdvecBatchDevice([m], [len(p2c)], [0.5], DEV)
    dev.set_instance(0, pos, vel, mdir, p2c)
    dev.enable_direct_hop(0.7)
    dev.disable_direct_hop()
    for _ in range(3):
        dev.step()
    torch.cuda.synchronize()
    P, M, C2 = pos.copy(), mdir.copy(), p2c.copy()
    OA.steps(P, vel, M, C2, m.c2c, m.c_pos_ll, 0.5, m.extents, 1.0, 3)
    got = dev.host_instance(0)
    np.testing.assert_array_equal(got["p2c"], C2)
    np.testing.assert_array_equal(got["pos"].view(np.uint64), P.view(np.uint64))


def test_check_grid_rejects_a_perturbed_mesh():
    """oppb_advec_check_grid counts every cell whose record differs from the periodic grid (a
    corner one ulp off, a neighbour changed).  An instance with a perturbed corner keeps reading
    its records, and its steps equal the oracle's on that mesh, next to a clean instance on the
    grid path."""
    specs = [(9, 7, 1.0, 0.5, 20, 0.8), (11, 6, 0.5, 0.3, 20, 1.2)]
    meshes = [AdvecMesh(nx, ny, cw) for nx, ny, cw, _, _, _ in specs]
    m = meshes[1]
    m.c_pos_ll[17, 0] = np.nextafter(m.c_pos_ll[17, 0], 10.0)
    host = [particles(mm, s[4], s[5], 70 + k) for k, (mm, s) in enumerate(zip(meshes, specs))]
    dev = AdvecBatchDevice(meshes, [len(h[3]) for h in host], [s[3] for s in specs], DEV)
    assert dev.grid_nx == [9, 0]
    for k, h in enumerate(host):
        dev.set_instance(k, *h)
    for _ in range(5):
        dev.step()
    torch.cuda.synchronize()
    ref, _ = _oracle(meshes, host, specs, 5)
    _assert_same(dev, ref)
    # A changed neighbour, checked on its own packed copy of the clean mesh.
    m2 = AdvecMesh(11, 6, 0.5)
    c2c = m2.c2c.copy()
    c2c[40, 1] = c2c[40, 0]
    cells = torch.zeros(m2.n_cells * 4, dtype=torch.float64, device=DEV)
    mism = torch.zeros(1, dtype=torch.int32, device=DEV)
    lib = L.load()
    for cc, want in ((m2.c2c, 0), (c2c, 1)):
        ll = torch.from_numpy(np.ascontiguousarray(m2.c_pos_ll.T)).to(DEV)
        nb = torch.from_numpy(np.ascontiguousarray(cc.T)).to(DEV)
        L.check("pack", lib.oppb_advec_pack_cells(cells.data_ptr(), 0, m2.n_cells, m2.n_cells, ll.data_ptr(),
                                                  nb.data_ptr(), None))
        L.check("check", lib.oppb_advec_check_grid(cells.data_ptr(), 0, m2.n_cells, m2.nx, m2.cell_width,
                                                   mism.data_ptr(), None))
        assert int(mism.item()) == want
    with pytest.raises(L.OppbError):  # n_cells not a multiple of nx
        L.check("check", lib.oppb_advec_check_grid(cells.data_ptr(), 0, m2.n_cells, 7, m2.cell_width,
                                                   mism.data_ptr(), None))


def test_verify_counts_particles_outside_their_cell():
    """oppb_advec_verify (verify_kernel, apps/app_neso_advection/kernels.h:115-151) against the
    same rule restated in numpy, on one instance after some steps with a few particles moved out
    of their cell by hand: on the box's edges a particle counts as inside, one ulp beyond it
    outside, and a cell whose global index is negative counts too."""
    specs = [(48, 40, 0.5, 0.5, 30, 0.5)]
    meshes, _, dev = _build(specs, seed0=77)
    for _ in range(5):
        dev.step()
    m = meshes[0]
    n = dev.counts[0]
    rng = np.random.default_rng(5)
    pos = dev.pos[:, :n].cpu().numpy().copy()
    p2c = dev.p2c[:n].cpu().numpy()
    w = m.cell_width
    ix, iy = p2c % m.nx, p2c // m.nx
    pick = rng.choice(n, 40, replace=False)
    pos[0, pick[:10]] = ix[pick[:10]] * w                                   # on the lower x edge: inside
    pos[1, pick[10:20]] = iy[pick[10:20]] * w + w                            # on the upper y edge: inside
    pos[0, pick[20:30]] = np.nextafter(ix[pick[20:30]] * w + w, np.inf)      # one ulp beyond: outside
    pos[1, pick[30:40]] = np.nextafter(iy[pick[30:40]] * w, -np.inf)         # one ulp below: outside
    dev.pos[:, :n] = torch.from_numpy(pos).to(DEV)
    gid = torch.arange(m.n_cells, dtype=torch.int32, device=DEV)
    gid[int(p2c[pick[0]])] = -1  # a negative global index counts as incorrect
    gidh = gid.cpu().numpy()
    g = gidh[p2c]
    giy, gix = g // m.nx, g - (g // m.nx) * m.nx
    giy = np.where(g < 0, -((-g) // m.nx), giy)  # C division truncates toward zero
    gix = g - giy * m.nx
    llx, lly = gix * w, giy * w
    bad = (gix < 0) | (giy < 0) | (pos[0] < llx) | (pos[0] > llx + w) | (pos[1] < lly) | (pos[1] > lly + w)
    count = torch.zeros(1, dtype=torch.int32, device=DEV)
    lib = L.load()
    for rep in range(2):  # added into the count, as the OPP_INC global is
        L.check("oppb_advec_verify", lib.oppb_advec_verify(dev.pos.data_ptr(), dev.capacity, dev.p2c.data_ptr(),
                                                           gid.data_ptr(), n, m.nx, w, count.data_ptr(), None))
        torch.cuda.synchronize()
        assert int(count.item()) == (rep + 1) * int(bad.sum())
    assert int(bad.sum()) >= 21  # the 20 moved out, and every particle of the cell with index -1


@pytest.mark.parametrize("size", [1, 31, 32, 33, 100_003])
def test_removal_bits_mark_removed_cells(size):
    """oppb_removal_bits: bit i of word i/32 is set exactly where p2c[i] is the removed marker."""
    rng = np.random.default_rng(size)
    p2c = rng.integers(0, 1000, size).astype(np.int32)
    p2c[rng.random(size) < 0.1] = L.REMOVED_CELL
    words = (size + 31) // 32
    bits = torch.full((words + 1,), -1, dtype=torch.int32, device=DEV)  # one guard word beyond
    d = torch.from_numpy(p2c).to(DEV)
    L.check("oppb_removal_bits", L.load().oppb_removal_bits(d.data_ptr(), size, bits.data_ptr(), None))
    got = bits.cpu().numpy().view(np.uint32)
    want = np.packbits((p2c == L.REMOVED_CELL).astype(np.uint8), bitorder="little")
    want = np.pad(want, (0, 4 * words - len(want))).view("<u4")
    np.testing.assert_array_equal(got[:words], want)
    assert got[words] == 0xFFFFFFFF
