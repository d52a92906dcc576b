"""FemPIC's node-side loops and field solve without a GPU: the library's host set-up against
the oracle's restatement (bit for bit), the oracle's node charge density and electric field
against the reference's generated seq loops (golden fixture always, live when oracle/_ref is
built), and the oracle's Newton step against a direct sparse solve of the same system."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oppb.fempic import HostMesh
from oppb.field import host_system
from oracle import field as F
from oracle import ref_runner as R

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("dims", [(4, 4, 8, 1.0, 1.0, 2.0), (10, 10, 40, 1.0, 1.0, 4.0), (3, 5, 4, 0.6, 1.1, 0.9)])
def test_setup_matches_oracle(dims):
    hm = HostMesh(*dims, solve_field=False)
    bnd = F.boundary_potential(hm.n_type, 1.0, 0.25)
    h = host_system(hm, bnd)
    o = F.FieldSystem(hm.n_pos, hm.n_type, bnd, hm.c2n)
    assert h["neq"] == o.neq > 0
    np.testing.assert_array_equal(h["node_to_eq"], o.node_to_eq)
    np.testing.assert_array_equal(h["k_rowptr"], o.k_rowptr)
    np.testing.assert_array_equal(h["k_col"], o.k_col)
    for name in ("det_j", "c_sd", "k_val", "f0"):
        np.testing.assert_array_equal(h[name].view(np.uint64), getattr(o, name).view(np.uint64), err_msg=name)
    # K symmetric and definite: with the reference's vertex order (volume > 0 after the ABCD ->
    # ADBC flip) detJ = -6V < 0 on every cell, so K is negative definite, which CG accepts;
    # the shape derivatives are barycentric gradients (summing to zero over a cell's vertices)
    import scipy.sparse as sp

    k = sp.csr_matrix((o.k_val, o.k_col, o.k_rowptr), shape=(o.neq, o.neq))
    assert abs(k - k.T).max() <= 1e-12 * abs(k).max()
    assert (o.det_j < 0).all() and (k.diagonal() < 0).all()
    np.testing.assert_allclose(o.c_sd.sum(axis=1), 0.0, atol=1e-9 * np.abs(o.c_sd).max())
    # K by diagonals: the box mesh's K lies on 15 diagonals (the form is kept when they hold at
    # most 1.5 nnz values, so not on the smallest mesh), and the diagonal form holds K's entries
    # at their offsets and zeros elsewhere
    off, dia = h["dia_off"], h["dia_val"]
    if 15 * h["neq"] > 1.5 * h["nnz"]:
        assert len(off) == 0
        return
    assert len(off) == 15 and np.all(np.diff(off) > 0) and dia.shape == (15, h["neq"])
    dense_from_dia = np.zeros_like(dia)
    rows = np.repeat(np.arange(h["neq"]), np.diff(h["k_rowptr"]))
    j = np.searchsorted(off, h["k_col"] - rows)
    assert np.all(off[j] == h["k_col"] - rows)
    dense_from_dia[j, rows] = h["k_val"]
    np.testing.assert_array_equal(dia.view(np.uint64), dense_from_dia.view(np.uint64))


def test_loops_match_reference_golden():
    z = np.load(GOLDEN / "field_loops_4x4x8.npz")
    den = F.node_charge_density(z["den"], z["n_vol"], float(z["spwt"]))
    np.testing.assert_array_equal(den.view(np.uint64), z["den_out"].view(np.uint64))
    ef = F.electric_field(z["c2n"], z["c_sd"], z["potential"])
    np.testing.assert_array_equal(ef.view(np.uint64), z["c_ef"].view(np.uint64))


@pytest.mark.skipif(not (R.REF_DIR / "field_ref_seq").exists(), reason="compiled reference not built")
def test_loops_match_live_reference():
    hm = HostMesh(10, 10, 40, 1.0, 1.0, 4.0, solve_field=False)
    fs = F.FieldSystem(hm.n_pos, hm.n_type, F.boundary_potential(hm.n_type, 1.0, 0.0), hm.c2n)
    rng = np.random.default_rng(3)
    den, pot = rng.random(hm.n_nodes) * 1e3, rng.normal(0.0, 2.0, hm.n_nodes)
    ref_den, ref_ef = F.run_reference(den, hm.n_vol, 2e2, hm.c2n, fs.c_sd, pot)
    np.testing.assert_array_equal(F.node_charge_density(den, hm.n_vol, 2e2).view(np.uint64), ref_den.view(np.uint64))
    np.testing.assert_array_equal(F.electric_field(hm.c2n, fs.c_sd, pot).view(np.uint64), ref_ef.view(np.uint64))


def _direct_newton_step(fs: F.FieldSystem, d_old, f1_old, ion_den, c: F.FieldConsts):
    """The same Newton step assembled in numpy and solved directly (scipy): every cell's
    8-point integral of the shape function is +detJ/2 for vertices 0..2 and -detJ/2 for 3."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    neq = fs.neq
    e_of = fs.node_to_eq
    t1 = np.zeros(neq)
    known = e_of >= 0
    t1[e_of[known]] = (c.qe / c.eps0) * (ion_den[known] + c.n0 * np.exp((d_old[e_of[known]] - c.phi0) / c.kte))
    t3 = -c.qe / c.eps0 * c.n0 * np.exp((d_old[:neq] - c.phi0) / c.kte) * (1 / c.kte)
    f1 = f1_old[:neq].copy()
    t2 = np.zeros(neq)
    sign = np.array([0.5, 0.5, 0.5, -0.5])
    for v in range(4):
        e = e_of[fs.c2n[:, v]]
        m = e >= 0
        np.add.at(f1, e[m], t1[e[m]] * fs.det_j[m] * sign[v])
        np.add.at(t2, e[m], t3[e[m]] * fs.det_j[m] * sign[v])
    k = sp.csr_matrix((fs.k_val, fs.k_col, fs.k_rowptr), shape=(neq, neq))
    b = k @ d_old[:neq] - fs.f0 - f1
    j = (k + sp.diags(-t2)).tocsc()
    y = spl.spsolve(j, b)
    return d_old[:neq] - y, f1


def test_oracle_newton_step_matches_direct_solve():
    hm = HostMesh(4, 4, 8, 1.0, 1.0, 2.0, solve_field=False)
    fs = F.FieldSystem(hm.n_pos, hm.n_type, F.boundary_potential(hm.n_type, 1.0, 0.0), hm.c2n)
    c = F.FieldConsts(n0=1.0, phi0=0.0, kte=1.0, qe=1.0, eps0=1.0)
    rng = np.random.default_rng(5)
    for step in range(3):  # F1 accumulates over the calls, as the reference's f1Local
        ion = rng.random(hm.n_nodes) * 2.0
        d_old, f1_old = fs.d.copy(), fs.f1.copy()
        pot, it, resid = fs.solve(ion, c)
        d_ref, f1_ref = _direct_newton_step(fs, d_old, f1_old, ion, c)
        assert 0 < it < c.max_iter and resid <= 1e-10
        np.testing.assert_allclose(fs.f1[:fs.neq], f1_ref, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(fs.d[:fs.neq], d_ref, rtol=1e-8, atol=1e-9 * np.abs(d_ref).max())
        known = fs.node_to_eq >= 0
        np.testing.assert_array_equal(pot[~known], fs.n_bnd_pot[~known])
        np.testing.assert_array_equal(pot[known], (fs.n_bnd_pot + 0.0)[known] + fs.d[fs.node_to_eq[known]])


def test_oracle_laplace_limit_matches_mesh_solver():
    """No electrons and no ions: one step gives the Laplace potential of the Dirichlet data,
    which the mesh builder also computes (its own assembly and CG)."""
    hm = HostMesh(6, 6, 12, 1.0, 1.0, 2.0)  # solves phi = 1 at z = 0, 0 at z = 2
    fs = F.FieldSystem(hm.n_pos, hm.n_type, F.boundary_potential(hm.n_type, 1.0, 0.0), hm.c2n)
    pot, it, resid = fs.solve(np.zeros(hm.n_nodes), F.FieldConsts(n0=0.0, phi0=0.0, kte=1.0, qe=1.0, eps0=1.0,
                                                                   rtol=1e-13, atol=0.0))
    assert resid <= 1e-13
    np.testing.assert_allclose(pot, hm.n_pot, rtol=0, atol=1e-9)
