"""CabanaPIC particle path without a GPU: the C oracle (oracle/cabana_oracle.c) against the
compiled reference seq backend — through the golden fixture it made
(tests/golden/make_golden_cabana.py) always, and live when oracle/_ref holds the build — and
the host-side mesh set-up against the reference's indexing rules."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oppb.cabana import Deck, HexMesh, synthetic_interp, two_stream
from oracle import cabana as OC
from oracle import ref_runner as R

GOLDEN = Path(__file__).resolve().parent / "golden" / "cabana_4x5x6.npz"


def _bits_equal(a, b, name):
    np.testing.assert_array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8), err_msg=name)


def test_oracle_matches_reference_golden():
    z = np.load(GOLDEN)
    mesh = HexMesh(*[int(v) for v in z["dims"]])
    pos, vel, streak, p2c = z["pos"].copy(), z["vel"].copy(), z["streak"].copy(), z["p2c"].copy()
    for _ in range(int(z["calls"])):
        acc = np.zeros((mesh.n_cells, 12))
        OC.move_deposit(pos, vel, streak, z["weight"], p2c, mesh.c2ngc, z["interp"], acc, float(z["qdt_2mc"]),
                        z["cdt_d"], float(z["qsp"]))
    for name, got in (("pos", pos), ("vel", vel), ("streak", streak), ("p2c", p2c), ("acc", acc)):
        _bits_equal(got, z["ref_" + name], name)
    assert (p2c != z["p2c"]).sum() > 1000  # the case walks across faces


@pytest.mark.skipif(not R.available("seq") or not (R.REF_DIR / "cabana_ref_seq").exists(),
                    reason="compiled reference absent")
@pytest.mark.parametrize("seed,scale", [(11, 0.5), (12, 3.0)])
def test_oracle_matches_reference_live(seed, scale):
    mesh = HexMesh(3, 4, 5)
    rng = np.random.default_rng(seed)
    interp = synthetic_interp(mesh, seed, e_scale=0.3, b_scale=0.5)
    n = 3000
    p2c = rng.choice(mesh.interior, n).astype(np.int32)
    pos = rng.uniform(-1, 1, (n, 3))
    vel = rng.normal(0, scale, (n, 3))
    streak, w = np.zeros((n, 3)), rng.uniform(0.1, 2.0, n)
    # particles exactly on faces and with zero momentum components
    pos[:50, 0] = 1.0
    pos[50:100, 2] = -1.0
    vel[100:150, 1] = 0.0
    cd = (1.3, 0.7, 2.1)
    ref = OC.run_reference("seq", mesh.c2ngc, interp, pos, vel, streak, w, p2c, -0.25, cd, -1.0, calls=2)
    acc = None
    for _ in range(2):
        acc = np.zeros((mesh.n_cells, 12))
        OC.move_deposit(pos, vel, streak, w, p2c, mesh.c2ngc, interp, acc, -0.25, np.array(cd), -1.0)
    for name, got in (("pos", pos), ("vel", vel), ("streak", streak), ("p2c", p2c), ("acc", acc)):
        _bits_equal(got, ref[name], name)


def test_hex_mesh_periodic_faces():
    m = HexMesh(3, 4, 5)
    gx, gy = 5, 6
    assert m.n_cells == 5 * 6 * 7
    interior = m.interior
    assert len(interior) == 3 * 4 * 5
    ghost = np.flatnonzero(m.ghost)
    np.testing.assert_array_equal(m.c2ngc[ghost], np.repeat(ghost[:, None], 6, axis=1))
    # every face neighbour of an interior cell is interior, and opposite faces invert
    assert m.ghost[m.c2ngc[interior]].sum() == 0
    for f in range(3):
        np.testing.assert_array_equal(m.c2ngc[m.c2ngc[interior, f], f + 3], interior)
    # VOXEL indexing: x fastest; interior (1,1,1) -> xd wraps to (3,1,1)
    c = 1 + gx * (1 + gy * 1)
    assert m.c2ngc[c, 0] == 3 + gx * (1 + gy * 1)
    assert m.c2ngc[c, 3] == 2 + gx * (1 + gy * 1)


def test_deck_and_two_stream():
    d = Deck(32, 32, 256, 1.0, 1.0, 8.0, nppc=400, courant_frac=0.5)
    assert abs(d.cdt_d[0] - 0.5 / np.sqrt(3.0)) < 1e-15
    assert abs(d.qdt_2mc + d.dt / 2) < 1e-18
    m = HexMesh(2, 2, 3)
    d2 = Deck(2, 2, 3, 1.0, 1.0, 1.5, nppc=10)
    pos, vel, streak, w, p2c = two_stream(m, d2, 0.2, 0.01, seed=0)
    assert len(p2c) == 12 * 10 and np.all(np.diff(p2c) >= 0)
    assert np.all(np.abs(pos) <= 1.0) and np.all(streak == 0)
    assert abs(np.mean(np.abs(vel[:, 2])) - 0.2 / np.sqrt(1 - 0.04)) < 0.01
