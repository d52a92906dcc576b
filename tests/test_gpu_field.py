"""FemPIC's node-side loops and field solve on the GPU (include/oppb_field.h) against the C
oracle: node charge density and electric field bit for bit (the oracle's loops equal the
reference's generated seq loops); the Newton step's potentials within 1e-8 of the oracle's
(both stop at ||r|| <= 1e-10 ||B||; the F1 sums use FP64 atomics, as the reference's device
kernels do); the field phase captured as a CUDA graph."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oppb.fempic import HostMesh
from oppb.field import FieldConstants, FieldDevice, boundary_potential
from oracle import field as F

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
UNIT = dict(n0=1.0, phi0=0.0, kte=1.0, qe=1.0, eps0=1.0)


def _close(gpu, ref, tol):
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.abs(gpu - ref).max() <= tol * scale, np.abs(gpu - ref).max() / scale


def test_node_density_and_field_bit_exact():
    hm = HostMesh(10, 10, 40, 1.0, 1.0, 4.0, solve_field=False)
    fd = FieldDevice(hm, DEV, boundary_potential(hm.n_type, 1.0, 0.0))
    rng = np.random.default_rng(2)
    den = rng.random(hm.n_nodes) * 1e3
    vol = torch.from_numpy(hm.n_vol).to(DEV)
    g = torch.from_numpy(den).to(DEV)
    fd.node_charge_density(g, vol, 2e2)
    np.testing.assert_array_equal(g.cpu().numpy().view(np.uint64),
                                  F.node_charge_density(den, hm.n_vol, 2e2).view(np.uint64))
    pot = rng.normal(0.0, 2.0, hm.n_nodes)
    fd.potential.copy_(torch.from_numpy(pot))
    ref = F.electric_field(hm.c2n, fd.c_sd, pot)
    ef3 = torch.zeros(hm.n_cells, 3, dtype=torch.float64, device=DEV)
    fd.electric_field(ef3, 3)
    np.testing.assert_array_equal(ef3.cpu().numpy().view(np.uint64), ref.view(np.uint64))
    ef4 = torch.full((hm.n_cells, 4), 7.0, dtype=torch.float64, device=DEV)  # the move's packed record
    fd.electric_field(ef4, 4)
    got = ef4.cpu().numpy()
    np.testing.assert_array_equal(got[:, :3].copy().view(np.uint64), ref.view(np.uint64))
    assert (got[:, 3] == 7.0).all()


@pytest.mark.parametrize("dims", [(4, 4, 8, 1.0, 1.0, 2.0), (10, 10, 40, 1.0, 1.0, 4.0)])
def test_newton_steps_match_oracle(dims):
    hm = HostMesh(*dims, solve_field=False)
    bnd = boundary_potential(hm.n_type, 1.0, 0.0)
    fd = FieldDevice(hm, DEV, bnd)
    fs = F.FieldSystem(hm.n_pos, hm.n_type, bnd, hm.c2n)
    cg = FieldConstants(**UNIT)
    co = F.FieldConsts(**UNIT)
    rng = np.random.default_rng(7)
    for step in range(3):  # F1 accumulates over the calls, as in the reference
        ion = rng.random(hm.n_nodes) * 2.0
        pot = fd.solve(torch.from_numpy(ion).to(DEV), cg).cpu().numpy()
        st = fd.status_host()
        pot_o, it_o, _ = fs.solve(ion, co)
        assert st.converged == 1 and st.resid <= 1e-10
        assert abs(st.iterations - it_o) <= 2, (st.iterations, it_o)
        _close(pot, pot_o, 1e-8)
        _close(fd.f1[:fd.neq].cpu().numpy(), fs.f1[:fs.neq], 1e-12)
        _close(fd.d[:fd.neq].cpu().numpy(), fs.d[:fs.neq], 1e-8)


def test_laplace_limit_matches_mesh_solver():
    hm = HostMesh(6, 6, 12, 1.0, 1.0, 2.0)
    fd = FieldDevice(hm, DEV, boundary_potential(hm.n_type, 1.0, 0.0))
    c = FieldConstants(n0=0.0, phi0=0.0, kte=1.0, qe=1.0, eps0=1.0, rtol=1e-13, atol=0.0)
    pot = fd.solve(torch.zeros(hm.n_nodes, dtype=torch.float64, device=DEV), c).cpu().numpy()
    assert fd.status_host().converged == 1
    np.testing.assert_allclose(pot, hm.n_pot, rtol=0, atol=1e-9)


def test_solve_repeats_and_graph_replay():
    """The CG reductions are deterministic; only the F1 / J-diagonal atomics can reorder, so
    two solves from the same state agree to rounding, and a captured graph of the field phase
    (density, potential, field) gives what the direct calls give."""
    hm = HostMesh(8, 8, 24, 1.0, 1.0, 3.0, solve_field=False)
    bnd = boundary_potential(hm.n_type, 1.0, 0.0)
    vol = torch.from_numpy(hm.n_vol).to(DEV)
    rng = np.random.default_rng(9)
    raw = torch.from_numpy(rng.random(hm.n_nodes) * 4.0).to(DEV)
    cg = FieldConstants(**UNIT)
    out = []
    for use_graph in (False, True, True):
        fd = FieldDevice(hm, DEV, bnd)
        den = raw.clone()
        ef = torch.zeros(hm.n_cells, 4, dtype=torch.float64, device=DEV)
        if use_graph:
            g = fd.capture(den, vol, 0.5, cg, ef, 4)
            den.copy_(raw)
            fd.d.zero_()
            fd.f1.zero_()
            g.replay()
        else:
            fd.node_charge_density(den, vol, 0.5)
            fd.solve(den, cg)
            fd.electric_field(ef, 4)
        torch.cuda.synchronize()
        assert fd.status_host().converged == 1
        out.append((fd.potential.cpu().numpy(), ef.cpu().numpy()))
    for pot, ef in out[1:]:
        _close(pot, out[0][0], 1e-12)
        _close(ef, out[0][1], 1e-11)


@pytest.mark.parametrize("dims", [(8, 8, 24, 1.0, 1.0, 3.0), (48, 48, 192, 1.0, 1.0, 4.0)])
def test_diagonal_form_equals_csr(dims):
    """The CG's products by diagonals add the same terms in the same order as the CSR rows, so
    one Newton step from the same state agrees with the CSR one as two CSR solves agree with
    each other (the F1 / J-diagonal atomics reorder between runs): same iteration count within
    one, potential within 1e-12."""
    hm = HostMesh(*dims, solve_field=False)
    bnd = boundary_potential(hm.n_type, 1.0, 0.0)
    rng = np.random.default_rng(3)
    ion = torch.from_numpy(rng.random(hm.n_nodes)).to(DEV)
    c = FieldConstants(n0=50.0, phi0=0.0, kte=1.0, qe=1.0, eps0=1.0)
    out = []
    for diag in (False, True):
        fd = FieldDevice(hm, DEV, bnd)
        assert len(fd.dia_off) == 15
        fd.set_diagonal_form(diag)
        pot = fd.solve(ion, c).cpu().numpy()
        st = fd.status_host()
        assert st.converged == 1
        out.append((pot, st.iterations))
    assert abs(out[0][1] - out[1][1]) <= 1 and out[0][1] > 10
    _close(out[1][0], out[0][0], 1e-12)


def test_full_size_solve_matches_oracle():
    """The 48x48x192-hex mesh (463,393 nodes): one Newton step against the oracle."""
    hm = HostMesh(48, 48, 192, 1.0, 1.0, 4.0, solve_field=False)
    bnd = boundary_potential(hm.n_type, 1.0, 0.0)
    fd = FieldDevice(hm, DEV, bnd)
    fs = F.FieldSystem(hm.n_pos, hm.n_type, bnd, hm.c2n)
    rng = np.random.default_rng(1)
    ion = rng.random(hm.n_nodes)
    c = dict(n0=50.0, phi0=0.0, kte=1.0, qe=1.0, eps0=1.0)  # Debye length ~ 7 cells
    pot = fd.solve(torch.from_numpy(ion).to(DEV), FieldConstants(**c)).cpu().numpy()
    st = fd.status_host()
    pot_o, it_o, _ = fs.solve(ion, F.FieldConsts(**c))
    assert st.converged == 1 and abs(st.iterations - it_o) <= 2
    _close(pot, pot_o, 1e-8)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_fempic_steps_with_field_phase_match_oracle(precision):
    """Whole steps with the field phase (the generated main loop's order): cells and counts
    equal to the oracle's, positions and fields within the CG tolerance's reach."""
    from oppb.fempic import FemPIC, injection_randoms, randoms_to_device
    from oracle import oracle as O

    hm = HostMesh(10, 10, 40, 1.0, 1.0, 4.0)
    hm_o = HostMesh(10, 10, 40, 1.0, 1.0, 4.0)  # the oracle rewrites its mesh's c_ef
    c = dict(n0=100.0, phi0=0.0, kte=1.0, qe=1.0, eps0=1.0)
    spwt = 100.0 * 4.0 / 20_000  # ion density ~ n0 once ~20k particles are in the box
    sim = FemPIC(hm, DEV, inject_per_step=2000, dt=0.05, precision=precision, field=FieldConstants(**c), spwt=spwt)
    fs = F.FieldSystem(hm_o.n_pos, hm_o.n_type, boundary_potential(hm_o.n_type, 1.0, 0.0), hm_o.c2n)
    orc = O.OracleFemPIC(hm_o, sim.dist_host, dt=0.05, mixed=(precision == "mixed"),
                         field=(fs, F.FieldConsts(**c), spwt, hm_o.n_vol))
    for s in range(12):
        rnd = injection_randoms(13, s, 2000, 0.1)
        g = sim.step(randoms_to_device(rnd, DEV))
        o = orc.step(rnd)
        assert (g["size"], g["removed"]) == (o["size"], o["removed"]), s
        assert sim.field.status_host().converged == 1
    got = sim.parts.host_aos()
    np.testing.assert_array_equal(got["p2c"], orc.p2c[:orc.size])
    # The mixed push rounds E to FP32: a field difference at the CG tolerance can move f32(E)
    # by one FP32 unit (6e-8 relative), so its positions agree to FP32 increments only.
    _close(got["pos"], orc.pos[:orc.size], 1e-9 if precision == "f64" else 1e-6)
    _close(sim.field.potential.cpu().numpy(), orc.potential, 1e-8)
    ef = sim.mesh.ef.view(-1, 4)[:, :3].cpu().numpy()
    _close(ef, hm_o.c_ef, 1e-7)
    assert np.abs(hm_o.c_ef - hm.c_ef).max() > 1e-3  # the field did change from the static one
