"""The deterministic deposit (OPPB_DEPOSIT_EXACT): node charges equal, bit for bit, the
correctly rounded sum of the weights cut to multiples of 2^-52 (the oracle's deposit_exact,
integer sums of the stored weights); they do not change when the particles are permuted, and whole FemPIC
steps repeat bit for bit.  Against the oracle's sequential FP64 sums they agree within 1e-12
of max(|q|, 1)."""
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


@pytest.fixture(autouse=True)
def exact_mode():
    L.set_tuning(deposit=L.DEPOSIT_EXACT)
    yield
    L.set_tuning(deposit=L.DEPOSIT_WARP_ATOMIC, replicas=8)


def _load(ps, pos, p2c):
    n = len(p2c)
    ps.size = n
    ps.pos[:, :n] = torch.from_numpy(pos.T.copy()).to(DEV)
    ps.p2c[0, :n] = torch.from_numpy(p2c).to(DEV)


def _move_deposit(dm, ps, kind):
    lib = L.load()
    charge = torch.zeros(dm.n_nodes, dtype=torch.float64, device=DEV)
    ws = torch.empty(lib.oppb_deposit_workspace_bytes(dm.n_nodes), dtype=torch.uint8, device=DEV)
    v = ps.view()
    if kind == "f64":
        rc = lib.oppb_move_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(), ps.status.data_ptr(), 4096,
                                       ws.data_ptr(), ws.numel(), None)
    else:
        rc = lib.oppb_move_deposit_mixed(C.byref(dm.s), C.byref(v), charge.data_ptr(), ps.status.data_ptr(), 4096,
                                         1e-5, ws.data_ptr(), ws.numel(), None)
    L.check("move_deposit", rc)
    torch.cuda.synchronize()
    return charge.cpu().numpy()


@pytest.mark.parametrize("kind", ["f64", "mixed"])
@pytest.mark.parametrize("n,seed", [(5000, 1), (300_001, 2)])
def test_exact_deposit_bit_exact_and_order_free(kind, n, seed):
    hm = mesh()
    dm = DeviceMesh(hm, DEV, mixed=(kind == "mixed"))
    pos, p2c = random_particles(hm, n, seed)
    ps = ParticleSet(DEV, n)
    _load(ps, pos, p2c)
    q = _move_deposit(dm, ps, kind)
    got = ps.host_aos()
    # the integer sums of the weights the kernel stored (FP64 lambdas, or FP32 ones widened)
    ref = O.deposit_exact(got["lc"], got["p2c"], hm.c2n, hm.n_nodes)
    np.testing.assert_array_equal(q.view(np.uint64), ref.view(np.uint64))
    # any particle order gives the same charges
    perm = np.random.default_rng(seed + 7).permutation(n)
    ps2 = ParticleSet(DEV, n)
    _load(ps2, pos[perm], p2c[perm])
    q2 = _move_deposit(dm, ps2, kind)
    np.testing.assert_array_equal(q2.view(np.uint64), q.view(np.uint64))
    if kind == "f64":  # the oracle's sequential FP64 sums, within their own rounding
        lc = np.zeros((n, 4))
        p2c_o = p2c.copy()
        O.move(pos, lc, p2c_o, hm.c2c, hm.c_vol, hm.c_det, n=n, max_hops=4096)
        np.testing.assert_array_equal(got["lc"].view(np.uint64), lc.view(np.uint64))
        keep = p2c_o != REMOVED
        seq = np.zeros(hm.n_nodes)
        O.deposit(np.ascontiguousarray(lc[keep]), np.ascontiguousarray(p2c_o[keep]), hm.c2n, seq)
        assert (np.abs(q - seq) / np.maximum(np.abs(seq), 1.0)).max() <= 1e-12


def test_exact_standalone_deposit_matches_fused():
    hm = mesh()
    dm = DeviceMesh(hm, DEV, mixed=False)
    pos, p2c = random_particles(hm, 20_000, 5)
    ps = ParticleSet(DEV, len(p2c))
    _load(ps, pos, p2c)
    q_fused = _move_deposit(dm, ps, "f64")
    lib = L.load()
    charge = torch.zeros(hm.n_nodes, dtype=torch.float64, device=DEV)
    ws = torch.empty(lib.oppb_deposit_workspace_bytes(hm.n_nodes), dtype=torch.uint8, device=DEV)
    v = ps.view()
    L.check("deposit", lib.oppb_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(), ws.data_ptr(), ws.numel(),
                                            None))
    np.testing.assert_array_equal(charge.cpu().numpy().view(np.uint64), q_fused.view(np.uint64))


def test_exact_deposit_needs_its_workspace():
    hm = mesh()
    dm = DeviceMesh(hm, DEV, mixed=False)
    pos, p2c = random_particles(hm, 1000, 6)
    ps = ParticleSet(DEV, len(p2c))
    _load(ps, pos, p2c)
    lib = L.load()
    charge = torch.zeros(hm.n_nodes, dtype=torch.float64, device=DEV)
    small = torch.empty(8 * hm.n_nodes, dtype=torch.uint8, device=DEV)
    v = ps.view()
    rc = lib.oppb_move_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(), ps.status.data_ptr(), 4096,
                                   small.data_ptr(), small.numel(), None)
    assert rc == L.OPPB_ERR_WORKSPACE


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_exact_fempic_steps_repeat_bit_for_bit(precision):
    """Two runs of the same steps (fused push, hole fills and sorts): node charges identical
    bit for bit at every step, which the atomics of the other deposit modes do not promise."""
    hm = mesh()
    runs = []
    for _ in range(2):
        sim = FemPIC(hm, DEV, inject_per_step=3000, precision=precision, fill="Sort_Periodic", fill_period=3)
        qs = []
        for s in range(8):
            sim.step(randoms_to_device(injection_randoms(21, s, 3000, 0.1), DEV))
            qs.append(sim.node_charge.cpu().numpy().copy())
        runs.append(qs)
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64))
