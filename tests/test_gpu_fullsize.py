"""Size-independent properties on the benchmark's 48x48x192-hex mesh (2,654,208 tets) with a few
million particles, where the oracle would take minutes: after each step every particle sits in
a valid cell with lambdas inside the inside-test band that sum to 1, the node charges add up to
the deposited weight (one per particle), a sort step leaves the cells in order, and the mixed
move takes the FP64 move's cell decisions from the same pushed state."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from oppb import _lib as L
from oppb.autotune import ParticleSnapshot
from oppb.fempic import FemPIC, HostMesh, injection_randoms, randoms_to_device

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
INJECT = 250_000


@pytest.fixture(scope="module")
def big_mesh():
    return HostMesh(48, 48, 192, 1.0, 1.0, 4.0)


def _run(hm, precision, steps):
    sim = FemPIC(hm, DEV, inject_per_step=INJECT, precision=precision, fill="Sort_Periodic", fill_period=10)
    outs = [sim.step(randoms_to_device(injection_randoms(31, s, INJECT, 0.1), DEV)) for s in range(steps)]
    return sim, outs


# The FP64 lambdas are the reference's expression coef * (((d0 - d1 x) + d2 y) - d3 z), each
# formed on its own with cancellation between cofactors of size ~1/h^2: their sum is 1 only to
# that expression's conditioning (errors up to ~1e-12 here), hence 1e-9; the mixed path's
# lambda_3 is 1 - lambda_0 - lambda_1 - lambda_2 in FP32 (or four FP64 values rounded to FP32).
@pytest.mark.parametrize("precision,sum_tol", [("f64", 1e-9), ("mixed", 1e-6)])
def test_fullsize_lambdas_and_charge_conservation(big_mesh, precision, sum_tol):
    sim, outs = _run(big_mesh, precision, 24)
    n = sim.parts.size
    assert n > 4_000_000 and outs[-1]["size"] == n
    p2c = sim.parts.p2c[0, :n]
    lc = sim.parts.lc[:, :n]
    assert bool(((p2c >= 0) & (p2c < big_mesh.n_cells)).all())
    band = 1e-10 if precision == "f64" else 1e-5  # the inside test's tolerance, the FP32 band
    assert float(lc.min()) > -band - 1e-12 and float(lc.max()) < 1.0 + band + 1e-12
    assert float((lc.sum(dim=0) - 1.0).abs().max()) <= sum_tol
    # The last step's deposit is the weight of every particle that stayed: sum q = sum lambda
    q_total = float(sim.node_charge.sum())
    lam_total = float(lc.sum())
    assert abs(q_total - lam_total) <= 1e-12 * n
    assert abs(q_total - n) <= sum_tol * n
    assert "sort" in [o["compaction"] for o in outs]  # Sort_Periodic ran at iteration 10 or 20


def test_fullsize_sort_leaves_cells_in_order(big_mesh):
    sim = FemPIC(big_mesh, DEV, inject_per_step=INJECT, precision="mixed", fill="Sort_Periodic", fill_period=10)
    sorted_steps = 0
    for s in range(25):
        out = sim.step(randoms_to_device(injection_randoms(37, s, INJECT, 0.1), DEV))
        if out["compaction"] == "sort":  # the particles are in cell order right after a sort
            p2c = sim.parts.p2c[0, :sim.parts.size]
            assert bool((p2c[1:] >= p2c[:-1]).all()), s
            sorted_steps += 1
        else:
            assert s % 10 != 0 or out["removed"] == 0, s
    assert sorted_steps >= 1


def test_fullsize_mixed_cells_equal_fp64(big_mesh):
    """From the same pushed state (the mixed steady state of 15 steps, pushed once), the mixed
    and the FP64 move + deposit reach the same cells and removals; charges agree within the
    FP32 weights' reach."""
    sim, _ = _run(big_mesh, "mixed", 15)
    sim.push()
    snap = ParticleSnapshot(sim)
    p, n = sim.parts, sim.parts.size
    res = {}
    for kind in ("mixed", "f64"):
        snap.restore()
        if kind == "mixed":
            sim.move()
        else:
            v, ws = p.view(), sim._deposit_ws()
            L.check("move", sim.lib.oppb_move_deposit_f64(C.byref(sim.mesh.s), C.byref(v), sim.node_charge.data_ptr(),
                                                          p.status.data_ptr(), sim.max_hops, ws.data_ptr(),
                                                          ws.numel(), None))
        torch.cuda.synchronize()
        st = p.status_host()
        assert st.error == 0
        res[kind] = (p.p2c[0, :n].clone(), sim.node_charge.clone(), st.remove_count, int(st.total_visits))
    (c_m, q_m, r_m, v_m), (c_f, q_f, r_f, v_f) = res["mixed"], res["f64"]
    assert torch.equal(c_m, c_f) and r_m == r_f and v_m == v_f
    assert float((q_m - q_f).abs().max() / q_f.abs().max()) <= 1e-5


@pytest.fixture(scope="module")
def steady_slice(big_mesh):
    """Config 2's steady state: 300 steps of 250,000 ions (Sort_Periodic every 10) on the
    2,654,208-tet mesh, one more injection and push, then a contiguous slice of 1,000,000
    particles from the middle of the set: host copies of its positions and start cells."""
    sim = FemPIC(big_mesh, DEV, inject_per_step=INJECT, fill="Sort_Periodic", fill_period=10, capacity=70_000_000)
    gen = torch.Generator(device=DEV)
    gen.manual_seed(0)
    rnd = torch.empty((5, INJECT), dtype=torch.float64, device=DEV)
    for _ in range(301):
        rnd[0:2].uniform_(0.0, 1.0, generator=gen)
        rnd[2:5].normal_(0.0, 0.1, generator=gen)
        if sim.iter < 300:
            sim.step(rnd)
        else:
            sim.inject(rnd)
            sim.push()
    n = sim.parts.size
    k = 1_000_000
    a = (n - k) // 2
    state = {"n": n, "pos": sim.parts.pos[:, a:a + k].T.contiguous().cpu().numpy(),
             "p2c": sim.parts.p2c[0, a:a + k].contiguous().cpu().numpy()}
    del sim
    torch.cuda.empty_cache()
    return state


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_fullsize_steady_state_slice_bit_exact(big_mesh, steady_slice, precision):
    """One steady-state move + deposit on 1,000,000 particles of config 2 (from a 57M-particle
    set): cells, removals and visit counts equal the oracle's; FP64 weights bit for bit (mixed:
    within 1e-5); node charges within 1e-12 relative (mixed: 1e-5 of the largest)."""
    from oppb.fempic import DeviceMesh, ParticleSet
    from oracle import oracle as O

    assert steady_slice["n"] > 50_000_000
    pos, p2c0 = steady_slice["pos"], steady_slice["p2c"]
    k = len(p2c0)
    dm = DeviceMesh(big_mesh, DEV, mixed=precision == "mixed")
    ps = ParticleSet(DEV, k)
    ps.size = k
    ps.pos[:, :k] = torch.from_numpy(pos.T.copy()).to(DEV)
    ps.p2c[0, :k] = torch.from_numpy(p2c0).to(DEV)
    charge = torch.zeros(big_mesh.n_nodes, dtype=torch.float64, device=DEV)
    nb = L.load().oppb_deposit_workspace_bytes(big_mesh.n_nodes)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=DEV)
    v = ps.view()
    if precision == "f64":
        rc = L.load().oppb_move_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(), ps.status.data_ptr(), 4096,
                                            ws.data_ptr(), nb, None)
    else:
        rc = L.load().oppb_move_deposit_mixed(C.byref(dm.s), C.byref(v), charge.data_ptr(), ps.status.data_ptr(),
                                              4096, 1e-5, ws.data_ptr(), nb, None)
    L.check("move_deposit", rc)
    torch.cuda.synchronize()
    st = ps.status_host()
    got = ps.host_aos()

    p2c = p2c0.copy()
    lc = np.zeros((k, 4))
    removed, visits, _ = O.move(pos, lc, p2c, big_mesh.c2c, big_mesh.c_vol, big_mesh.c_det, n=k)
    keep = p2c != O.REMOVED
    q = np.zeros(big_mesh.n_nodes)
    O.deposit(np.ascontiguousarray(lc[keep]), np.ascontiguousarray(p2c[keep]), big_mesh.c2n, q)

    assert st.error == 0 and st.remove_count == removed and int(st.total_visits) == visits
    np.testing.assert_array_equal(got["p2c"], p2c)
    qg = charge.cpu().numpy()
    if precision == "f64":
        np.testing.assert_array_equal(got["lc"][keep].view(np.uint64), lc[keep].view(np.uint64))
        assert (np.abs(qg - q) / np.maximum(np.abs(q), 1.0)).max() <= 1e-12
    else:
        assert np.abs(got["lc"][keep] - lc[keep]).max() <= 1e-5
        assert np.abs(qg - q).max() / np.abs(q).max() <= 1e-5
    assert visits > k
