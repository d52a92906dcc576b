"""Host set-up of the FemPIC mesh: the reference's own mesh check (each tet centroid lies
in its tet, minifempic_funcs.h:456-457), face-neighbour symmetry, volumes, inlet, field."""
from __future__ import annotations

import numpy as np

from helpers import mesh


def test_volumes_and_centroids():
    hm = mesh()
    assert hm.n_cells == 24000 and hm.n_nodes == 4961 and hm.n_ifaces == 200
    assert (hm.c_vol > 0).all()
    assert abs(hm.c_vol.sum() - 4.0) < 1e-12
    det = hm.c_det.reshape(-1, 4, 4)
    x = hm.c_centroid
    lam = ((1.0 / 6.0) / hm.c_vol)[:, None] * (det[:, :, 0] - det[:, :, 1] * x[:, 0:1] + det[:, :, 2] * x[:, 1:2]
                                               - det[:, :, 3] * x[:, 2:3])
    assert np.abs(lam - 0.25).max() < 1e-9


def test_face_neighbours_symmetric_and_share_three_nodes():
    hm = mesh()
    c2c, c2n = hm.c2c, hm.c2n
    for c in range(0, hm.n_cells, 37):
        for v in range(4):
            nb = c2c[c, v]
            if nb < 0:
                continue
            assert c in c2c[nb]
            face = set(c2n[c]) - {c2n[c, v]}
            assert face <= set(c2n[nb])
    # boundary faces: 2 per hex face on the box surface
    assert (c2c < 0).sum() == 2 * 2 * (10 * 10 + 10 * 40 + 10 * 40)


def test_inlet_faces_and_distribution():
    hm = mesh()
    assert np.allclose(hm.if_norm, [0.0, 0.0, 1.0])
    assert np.allclose(hm.if_area, 0.005)
    assert (hm.n_pos[hm.if2n][:, :, 2] == 0.0).all()
    # the inlet cell holds the face's three nodes
    for f in range(hm.n_ifaces):
        assert set(hm.if2n[f]) <= set(hm.c2n[hm.if2c[f]])
    d = hm.inject_distribution(2000)
    assert d[-1] == 2000 and (np.diff(np.r_[0, d]) == 10).all()
    d2 = hm.inject_distribution(12345)
    assert d2[-1] == 12345 and (np.diff(np.r_[0, d2]) > 0).all()


def test_static_field_is_uniform():
    hm = mesh()
    assert hm.cg_resid < 1e-12
    np.testing.assert_allclose(hm.c_ef[:, 2], 0.25, rtol=1e-10)
    assert np.abs(hm.c_ef[:, :2]).max() < 1e-10
    np.testing.assert_allclose(hm.n_pot, 1.0 - hm.n_pos[:, 2] / 4.0, atol=1e-12)
