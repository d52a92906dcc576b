"""NESO-advection particle path without a GPU: the C oracle (oracle/advec_oracle.c) against the
compiled reference seq backend — through its golden fixture (tests/golden/make_golden_advec.py)
always, and live when oracle/_ref holds the build — and the mesh set-up's neighbour rules."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from helpers import advec_edge_particles
from oppb.advec import AdvecMesh, particles
from oracle import advec as OA
from oracle import ref_runner as R

GOLDEN = Path(__file__).resolve().parent / "golden" / "advec_13x9.npz"
GOLDEN_DH = Path(__file__).resolve().parent / "golden" / "advec_dh_9x8.npz"
REMOVED = 2147483647


def test_oracle_matches_reference_golden():
    z = np.load(GOLDEN)
    m = AdvecMesh(int(z["nx"]), int(z["ny"]), float(z["cell_width"]))
    pos, mdir, p2c = z["pos"].copy(), z["mdir"].copy(), z["p2c"].copy()
    OA.steps(pos, z["vel"], mdir, p2c, m.c2c, m.c_pos_ll, float(z["dt"]), m.extents, m.cell_width, int(z["steps"]))
    np.testing.assert_array_equal(pos.view(np.uint64), z["ref_pos"].view(np.uint64))
    np.testing.assert_array_equal(mdir, z["ref_mdir"])
    np.testing.assert_array_equal(p2c, z["ref_p2c"])
    assert (p2c != z["p2c"]).mean() > 0.5


@pytest.mark.skipif(not (R.REF_DIR / "advec_ref_seq").exists(), reason="compiled reference absent")
@pytest.mark.parametrize("nx,ny,cw,dt,v_sd,steps", [(5, 17, 1.0, 0.5, 0.4, 12), (31, 6, 0.25, 0.9, 3.0, 5)])
def test_oracle_matches_reference_live(nx, ny, cw, dt, v_sd, steps):
    # The reference's wrap (n = int(|x| + 2) extents added before FMOD) lands in [0, extent)
    # only for extents >= 1; below that a position stays outside the mesh and its unbounded
    # hop loop never ends, so every case here keeps both extents >= 1.
    m = AdvecMesh(nx, ny, cw)
    pos, vel, mdir, p2c = particles(m, 20, v_sd, nx * 100 + ny)
    vel[:10] = 0.0  # resting particles
    pos[10:20, 0] = m.c_pos_ll[p2c[10:20], 0]  # on the lower-left edge of their cell
    ref = OA.run_reference("seq", nx, ny, cw, dt, pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, steps)
    OA.steps(pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, dt, m.extents, cw, steps)
    np.testing.assert_array_equal(pos.view(np.uint64), ref["pos"].view(np.uint64))
    np.testing.assert_array_equal(mdir, ref["mdir"])
    np.testing.assert_array_equal(p2c, ref["p2c"])


def test_oracle_direct_hop_matches_reference_golden():
    """The global move on (opp_init_direct_hop_cg, grid spacing 0.7 over unit cells): the
    oracle's grid and structured map equal the reference's, and so do 7 steps whose walks start
    from the seed, with particles on cell edges that the seed moves to the neighbouring cell."""
    z = np.load(GOLDEN_DH)
    cw = float(z["cell_width"])
    m = AdvecMesh(int(z["nx"]), int(z["ny"]), cw)
    g = OA.dh_build(m.c_pos_ll, cw, m.extents, float(z["grid_spacing"]), (2 * cw, 2 * cw, 0.0))
    np.testing.assert_array_equal(g.dims, z["ref_dims"])
    np.testing.assert_array_equal(g.box.view(np.uint64), z["ref_box"].view(np.uint64))
    np.testing.assert_array_equal(g.map, z["ref_map"])
    assert (g.map == REMOVED).any() and (g.map != REMOVED).any()
    pos, mdir, p2c = z["pos"].copy(), z["mdir"].copy(), z["p2c"].copy()
    _, removed = OA.steps_dh(pos, z["vel"], mdir, p2c, m.c2c, m.c_pos_ll, float(z["dt"]), m.extents, cw,
                             int(z["steps"]), g)
    np.testing.assert_array_equal(pos.view(np.uint64), z["ref_pos"].view(np.uint64))
    np.testing.assert_array_equal(mdir, z["ref_mdir"])
    np.testing.assert_array_equal(p2c, z["ref_p2c"])
    assert removed == 0
    # without the seed the edge particles end in other cells
    pos2, mdir2, p2c2 = z["pos"].copy(), z["mdir"].copy(), z["p2c"].copy()
    OA.steps(pos2, z["vel"], mdir2, p2c2, m.c2c, m.c_pos_ll, float(z["dt"]), m.extents, cw, int(z["steps"]))
    assert (p2c2 != p2c).sum() > 20


@pytest.mark.skipif(not (R.REF_DIR / "advec_ref_seq").exists(), reason="compiled reference absent")
@pytest.mark.parametrize("nx,ny,cw,gs", [(13, 9, 0.5, 0.5), (7, 11, 1.0, 0.3), (10, 6, 0.25, 0.4), (12, 12, 1.0, 1.0),
                                         (5, 19, 0.8, 1.9)])
def test_oracle_direct_hop_matches_reference_live(nx, ny, cw, gs):
    m = AdvecMesh(nx, ny, cw)
    pos, vel, mdir, p2c = advec_edge_particles(m, 12, 0.6, nx * 31 + ny)
    ref = OA.run_reference("seq", nx, ny, cw, 0.45, pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, 6, dh_spacing=gs)
    g = OA.dh_build(m.c_pos_ll, cw, m.extents, gs, (2 * cw, 2 * cw, 0.0))
    np.testing.assert_array_equal(g.dims, ref["dims"])
    np.testing.assert_array_equal(g.box.view(np.uint64), ref["box"].view(np.uint64))
    np.testing.assert_array_equal(g.map, ref["map"])
    OA.steps_dh(pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, 0.45, m.extents, cw, 6, g)
    np.testing.assert_array_equal(pos.view(np.uint64), ref["pos"].view(np.uint64))
    np.testing.assert_array_equal(mdir, ref["mdir"])
    np.testing.assert_array_equal(p2c, ref["p2c"])


def test_oracle_direct_hop_seed_removes_outside_the_grid():
    """The CUDA rule: a box coordinate at or past the grid's count on either axis (or a box
    without a cell) removes the particle; negative offsets truncate to box 0; removed stay."""
    m = AdvecMesh(6, 5, 1.0)
    g = OA.dh_build(m.c_pos_ll, 1.0, m.extents, 0.5, (2.0, 2.0, 0.0))
    pos = np.array([[0.5, 0.5], [1e9, 0.5], [0.5, 1e9], [-1e9, 2.5], [5.2, 4.9], [3.0, 3.0]])
    p2c = np.array([0, 0, 0, 0, 0, REMOVED], np.int32)
    removed = OA.dh_seed(pos, p2c, g)
    assert p2c[0] == 0 and p2c[1] == REMOVED and p2c[2] == REMOVED and p2c[5] == REMOVED
    assert p2c[4] == 5 + 6 * 4
    # x = -1e9 truncates to box 0 in x, a box left of the mesh: no cell
    assert p2c[3] == REMOVED and removed == 3


def test_mesh_neighbours_periodic():
    m = AdvecMesh(4, 3, 0.5)
    assert m.n_cells == 12
    np.testing.assert_array_equal(m.c2c[0], [3, 1, 8, 4])  # xd wraps to x=3, yd wraps to y=2
    for a, b in ((0, 1), (2, 3)):  # opposite directions invert
        np.testing.assert_array_equal(m.c2c[m.c2c[:, a], b], np.arange(12))
    np.testing.assert_allclose(m.c_pos_ll[5], [0.5, 0.5])
    assert m.extents == (2.0, 1.5)


def test_shard_instances_lpt():
    from oppb.advec import shard_instances

    rng = np.random.default_rng(4)
    w = [int(x) for x in rng.integers(1, 10**6, 64)]
    for ranks in (1, 2, 3, 4, 8, 64, 70):
        sh = shard_instances(w, ranks)
        assert len(sh) == ranks
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(w)))  # a partition of the instances
        assert all(s == sorted(s) for s in sh)
        loads = [sum(w[i] for i in s) for s in sh]
        assert max(loads) <= sum(w) / ranks + max(w)  # the LPT bound
    assert shard_instances(w, 1) == [list(range(64))]
    # by hand: 7 (#1) -> r0, 5 (#3) -> r1, 4 (#2) -> r1 (5 < 7), 3 (#0) -> r0 (7 < 9),
    # 3 (#4) -> r1 (9 < 10); loads 10 and 12
    assert shard_instances([3, 7, 4, 5, 3], 2) == [[0, 1], [2, 3, 4]]
    assert shard_instances([5, 5], 2) == [[0], [1]]  # ties: lower index to lower rank
    with pytest.raises(ValueError):
        shard_instances(w, 0)
