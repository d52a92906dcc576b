"""NESO-advection particle path without a GPU: the C oracle (oracle/advec_oracle.c) against the
compiled reference seq backend — through its golden fixture (tests/golden/make_golden_advec.py)
always, and live when oracle/_ref holds the build — and the mesh set-up's neighbour rules."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oppb.advec import AdvecMesh, particles
from oracle import advec as OA
from oracle import ref_runner as R

GOLDEN = Path(__file__).resolve().parent / "golden" / "advec_13x9.npz"


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
