"""Block shapes of the one-lane move kernels with the warp-grouped deposit (oppb_tuning.move_block
= 128, 256 or 512 threads per CTA).  The shape changes which CTA a particle is walked in, and
so the order of the FP64 atomics and the node-sum copy a CTA adds into, nothing else: cells,
weights, removal bitmap and status counts equal the default shape's bit for bit (and the
oracle's for FP64), node charges within 1e-12 relative; the device-count launches of
graph-captured steps included, with ragged particle counts."""
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
CHARGE_RTOL = 1e-12


@pytest.fixture(params=[128, 512])
def block(request):
    L.set_tuning(deposit=L.DEPOSIT_WARP_ATOMIC, move_lanes=1, move_stage=0, move_block=request.param)
    yield request.param
    L.set_tuning(move_block=256)


def _charge_close(a: np.ndarray, b: np.ndarray) -> None:
    err = np.abs(a - b) / np.maximum(np.abs(b), 1.0)
    assert err.max() <= CHARGE_RTOL, f"node charge max rel err {err.max():.3e}"


def _move_deposit(precision, hm, dm, pos, p2c):
    n = len(p2c)
    ps = ParticleSet(DEV, n)
    ps.increase(n)
    ps.size = n
    ps.pos[:, :n] = torch.from_numpy(pos.T.copy()).to(DEV)
    ps.p2c[0, :n] = torch.from_numpy(p2c).to(DEV)
    charge = torch.zeros(hm.n_nodes, dtype=torch.float64, device=DEV)
    ws = torch.empty(max(1, L.load().oppb_deposit_workspace_bytes(hm.n_nodes)), dtype=torch.uint8, device=DEV)
    v = ps.view()
    if precision == "f64":
        rc = L.load().oppb_move_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(), ps.status.data_ptr(), 4096,
                                            ws.data_ptr(), ws.numel(), None)
    else:
        rc = L.load().oppb_move_deposit_mixed(C.byref(dm.s), C.byref(v), charge.data_ptr(), ps.status.data_ptr(),
                                              4096, 1e-5, ws.data_ptr(), ws.numel(), None)
    L.check("move_deposit", rc)
    torch.cuda.synchronize()
    st = ps.status_host()
    got = ps.host_aos()
    bits = ps.bits.cpu().numpy().copy()
    return st, got, bits, charge.cpu().numpy()


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("n,seed", [(1, 0), (129, 1), (513, 2), (300_001, 3)])
def test_block_shape_equals_default(block, precision, n, seed):
    hm = mesh()
    dm = DeviceMesh(hm, DEV, mixed=precision == "mixed")
    pos, p2c = random_particles(hm, n, seed)
    st, got, bits, charge = _move_deposit(precision, hm, dm, pos, p2c)
    L.set_tuning(move_block=256)
    st0, got0, bits0, charge0 = _move_deposit(precision, hm, dm, pos, p2c)
    assert st.error == 0 and st0.error == 0
    assert (st.remove_count, st.total_visits, st.max_visits, st.recheck_count) == \
        (st0.remove_count, st0.total_visits, st0.max_visits, st0.recheck_count)
    np.testing.assert_array_equal(got["p2c"], got0["p2c"])
    np.testing.assert_array_equal(got["lc"].view(np.uint64), got0["lc"].view(np.uint64))
    np.testing.assert_array_equal(bits, bits0)
    _charge_close(charge, charge0)
    if precision == "f64":  # and the oracle's
        lc = np.zeros((n, 4))
        p2c_o = p2c.copy()
        rc, visits, _ = O.move(pos, lc, p2c_o, hm.c2c, hm.c_vol, hm.c_det, n=n, max_hops=4096)
        assert st.remove_count == rc and int(st.total_visits) == visits
        np.testing.assert_array_equal(got["p2c"], p2c_o)
        np.testing.assert_array_equal(got["lc"].view(np.uint64), lc.view(np.uint64))
        keep = p2c_o != REMOVED
        ref = np.zeros(hm.n_nodes)
        O.deposit(np.ascontiguousarray(lc[keep]), np.ascontiguousarray(p2c_o[keep]), hm.c2n, ref)
        _charge_close(charge, ref)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_block_shape_graph_steps_equal_default_direct_steps(block, precision):
    """40 graph-replayed steps (push fused into the device-count move, Sort_Periodic every 5) at
    this block shape against 40 direct steps at 256 threads, same tables."""
    hm = mesh()
    kw = dict(inject_per_step=2000, precision=precision, fill="Sort_Periodic", fill_period=5)
    graphed = FemPIC(hm, DEV, **kw)
    L.set_tuning(move_block=256)
    direct = FemPIC(hm, DEV, **kw)
    for r in range(4):
        tabs = [randoms_to_device(injection_randoms(12, r * 10 + k, 2000, 0.1), DEV) for k in range(10)]
        L.set_tuning(move_block=256)
        want = [direct.step(t) for t in tabs]
        L.set_tuning(move_block=block)
        got = graphed.run_graph(tabs)
        key = ("size_before_move", "removed", "size", "visits", "max_visits", "rechecks")
        assert [tuple(a[x] for x in key) for a in want] == [tuple(b[x] for x in key) for b in got], r
    a, b = direct.parts.host_aos(), graphed.parts.host_aos()
    for name in ("p2c", "pos", "vel", "lc"):
        np.testing.assert_array_equal(a[name].view(np.uint8), b[name].view(np.uint8), err_msg=name)
    _charge_close(graphed.node_charge.cpu().numpy(), direct.node_charge.cpu().numpy())
    assert direct.parts.size > 50_000


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_tune_block_leaves_state_and_picks_a_candidate(precision):
    from oppb.autotune import BLOCK_CANDIDATES, tune_block

    L.set_tuning(deposit=L.DEPOSIT_WARP_ATOMIC, move_lanes=1, move_stage=0, move_block=256)
    hm = mesh()
    sim = FemPIC(hm, DEV, inject_per_step=2000, precision=precision, fill="Sort_Periodic", fill_period=4)
    for k in range(6):
        sim.step(randoms_to_device(injection_randoms(3, k, 2000, 0.1), DEV))
    before = sim.parts.host_aos()
    try:
        res = tune_block(sim, reps=1)
        t = L.Tuning()
        L.load().oppb_get_tuning(C.byref(t))
        assert res.choice in BLOCK_CANDIDATES and set(res.times_ms) == set(BLOCK_CANDIDATES)
        assert t.move_block == res.choice
    finally:
        L.set_tuning(move_block=256)
    after = sim.parts.host_aos()
    for name in before:
        np.testing.assert_array_equal(before[name].view(np.uint8), after[name].view(np.uint8), err_msg=name)
