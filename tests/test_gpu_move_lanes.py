"""The FP64 move's variants: two lanes per particle (oppb_tuning.move_lanes = 2, compiled for 8
or 5 resident CTAs per SM), one lane with each visit's cell record staged into shared memory
by bulk asynchronous copies (move_stage = 1), and the walk on the mixed path's FP32 records with
the FP64 lambdas evaluated at the last cell (move_walk32 = 1).  Cells, weights, removals, visit counts and the
removal bitmap bit-exact against the oracle, as the default kernel; node charges within 1e-12
relative (FP64 atomics), and bit for bit equal to the default kernel's in the deterministic
deposit; the fused push, the device-count launch and the error paths (hop limit, bad cell)
included."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from helpers import REMOVED, mesh, random_particles
from oppb import _lib as L
from oppb.fempic import DeviceMesh, FemPIC, ParticleSet, injection_randoms, randoms_to_device
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


DEFAULT = (1, 8, 0, 0)  # (move_lanes, move_occupancy, move_stage, move_walk32)


def _set(v):
    L.set_tuning(move_lanes=v[0], move_occupancy=v[1], move_stage=v[2], move_walk32=v[3])


@pytest.fixture(params=[(1, 8, 1, 0), (2, 8, 0, 0), (2, 5, 0, 0), (1, 8, 0, 1), (1, 8, 0, 2)],
                ids=["staged", "pair-occ8", "pair-occ5", "walk32-occ8", "walk32-occ6"])
def pair_lanes(request):
    _set(request.param)
    yield request.param
    _set(DEFAULT)


def _particles(hm, n, seed):
    pos, p2c = random_particles(hm, n, seed)
    ps = ParticleSet(DEV, n)
    ps.increase(n)
    ps.size = n
    ps.pos[:, :n] = torch.from_numpy(pos.T.copy()).to(DEV)
    ps.p2c[0, :n] = torch.from_numpy(p2c).to(DEV)
    return pos, p2c, ps


def _move_deposit(dm, ps, hm, charge):
    ws = torch.empty(max(1, L.load().oppb_deposit_workspace_bytes(hm.n_nodes)), dtype=torch.uint8, device=DEV)
    v = ps.view()
    return L.load().oppb_move_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(), ps.status.data_ptr(), 4096,
                                          ws.data_ptr(), ws.numel(), None)


@pytest.mark.parametrize("deposit", [L.DEPOSIT_WARP_ATOMIC, L.DEPOSIT_CTA_TABLE])
@pytest.mark.parametrize("n,seed", [(1, 0), (257, 1), (5000, 4), (300_001, 5)])
def test_pair_move_deposit_matches_oracle(pair_lanes, deposit, n, seed):
    L.set_tuning(deposit=deposit)
    try:
        hm = mesh()
        dm = DeviceMesh(hm, DEV, mixed=True)
        pos, p2c, ps = _particles(hm, n, seed)
        charge = torch.zeros(hm.n_nodes, dtype=torch.float64, device=DEV)
        L.check("move_deposit", _move_deposit(dm, ps, hm, charge))
        torch.cuda.synchronize()
    finally:
        L.set_tuning(deposit=L.DEPOSIT_WARP_ATOMIC)
    st = ps.status_host()
    lc = np.zeros((n, 4))
    p2c_o = p2c.copy()
    rc, visits, per = O.move(pos, lc, p2c_o, hm.c2c, hm.c_vol, hm.c_det, n=n, max_hops=4096)
    keep = p2c_o != REMOVED
    ref = np.zeros(hm.n_nodes)
    O.deposit(np.ascontiguousarray(lc[keep]), np.ascontiguousarray(p2c_o[keep]), hm.c2n, ref)
    assert st.error == 0 and st.remove_count == rc and int(st.total_visits) == visits
    assert st.max_visits == int(per.max())
    got = ps.host_aos()
    np.testing.assert_array_equal(got["p2c"], p2c_o)
    np.testing.assert_array_equal(got["lc"].view(np.uint64), lc.view(np.uint64))
    err = np.abs(charge.cpu().numpy() - ref) / np.maximum(np.abs(ref), 1.0)
    assert err.max() <= 1e-12
    bits = ps.bits.cpu().numpy().view(np.uint32)
    rebuilt = np.flatnonzero(np.unpackbits(bits.view(np.uint8), bitorder="little")[:n])
    np.testing.assert_array_equal(rebuilt, np.flatnonzero(p2c_o == REMOVED))


def test_pair_exact_deposit_equals_one_lane_bit_for_bit(pair_lanes):
    """OPPB_DEPOSIT_EXACT sums integers: the node charges of the lane-pair kernel equal the
    one-lane kernel's bit for bit on the same particles."""
    hm = mesh()
    dm = DeviceMesh(hm, DEV, mixed=True)
    out = {}
    for variant in (DEFAULT, pair_lanes):
        L.set_tuning(deposit=L.DEPOSIT_EXACT)
        _set(variant)
        try:
            _, _, ps = _particles(hm, 200_000, 9)
            charge = torch.zeros(hm.n_nodes, dtype=torch.float64, device=DEV)
            L.check("move_deposit", _move_deposit(dm, ps, hm, charge))
            torch.cuda.synchronize()
        finally:
            L.set_tuning(deposit=L.DEPOSIT_WARP_ATOMIC)
            _set(pair_lanes)
        out[variant] = charge.cpu().numpy()
    np.testing.assert_array_equal(out[DEFAULT].view(np.uint64), out[pair_lanes].view(np.uint64))


def test_pair_fempic_steps_match_oracle(pair_lanes):
    """Config 1 through FemPIC with the push fused into the lane-pair kernel: 200 steps of
    2,000 ions, Sort_Periodic every 10, against the oracle."""
    hm = mesh()
    sim = FemPIC(hm, DEV, inject_per_step=2000, fill="Sort_Periodic", fill_period=10)
    orc = O.OracleFemPIC(hm, sim.dist_host, fill="Sort_Periodic", fill_period=10)
    for s in range(200):
        rnd = injection_randoms(21, s, 2000, 0.1)
        g = sim.step(randoms_to_device(rnd, DEV))
        o = orc.step(rnd)
        assert (g["size"], g["removed"], g["visits"]) == (o["size"], o["removed"], o["visits"]), s
    got, n = sim.parts.host_aos(), orc.size
    np.testing.assert_array_equal(got["p2c"], orc.p2c[:n])
    for name in ("pos", "vel", "lc"):
        np.testing.assert_array_equal(got[name].view(np.uint64), getattr(orc, name)[:n].view(np.uint64), err_msg=name)
    err = np.abs(sim.node_charge.cpu().numpy() - orc.node_charge) / np.maximum(np.abs(orc.node_charge), 1.0)
    assert err.max() <= 1e-12 and n > 100_000


def test_pair_graph_steps_equal_direct(pair_lanes):
    """The device-count launch of the lane-pair kernel inside graph-captured steps."""
    hm = mesh()
    direct = FemPIC(hm, DEV, inject_per_step=2000, fill="Sort_Periodic", fill_period=5)
    graphed = FemPIC(hm, DEV, inject_per_step=2000, fill="Sort_Periodic", fill_period=5)
    for r in range(4):
        tabs = [randoms_to_device(injection_randoms(8, r * 10 + k, 2000, 0.1), DEV) for k in range(10)]
        want = [direct.step(t) for t in tabs]
        got = graphed.run_graph(tabs)
        assert [(a["size"], a["visits"]) for a in want] == [(b["size"], b["visits"]) for b in got]
    a, b = direct.parts.host_aos(), graphed.parts.host_aos()
    for name in ("p2c", "pos", "vel", "lc"):
        np.testing.assert_array_equal(a[name].view(np.uint8), b[name].view(np.uint8), err_msg=name)


def test_pair_errors_reported(pair_lanes):
    """A bad start cell and the hop limit raise their error word with the particle index."""
    hm = mesh()
    dm = DeviceMesh(hm, DEV, mixed=True)
    pos, p2c, ps = _particles(hm, 600, 3)
    ps.p2c[0, 417] = hm.n_cells + 5
    charge = torch.zeros(hm.n_nodes, dtype=torch.float64, device=DEV)
    L.check("move_deposit", _move_deposit(dm, ps, hm, charge))
    st = ps.status_host()
    assert st.error == L.OPPB_ERR_CELL_RANGE and st.error_index == 417
    ps2 = ParticleSet(DEV, 1)
    ps2.increase(1)
    ps2.size = 1
    ps2.pos[:, :1] = torch.tensor([[0.95], [0.95], [3.9]], dtype=torch.float64, device=DEV)
    ps2.p2c[0, 0] = 0
    ws = torch.empty(max(1, L.load().oppb_deposit_workspace_bytes(hm.n_nodes)), dtype=torch.uint8, device=DEV)
    v = ps2.view()
    L.check("move", L.load().oppb_move_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(),
                                                   ps2.status.data_ptr(), 3, ws.data_ptr(), ws.numel(), None))
    st = ps2.status_host()
    assert st.error == L.OPPB_ERR_HOP_LIMIT and st.error_index == 0
