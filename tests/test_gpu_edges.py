"""Edge cases of the particle entry points: an empty particle set through every launcher (each
returns OPPB_OK, leaves the move status and the node charges at zero and launches nothing
that writes), a cell sort whose keys need a fourth radix pass and one whose keys fit one
bit, hole fills whose holes sit only at the tail or only at the head, and one over more bitmap
blocks than one pass of the single-block scan takes."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from helpers import REMOVED, mesh
from oppb import _lib as L
from oppb.fempic import DeviceMesh, ParticleSet, randoms_to_device, injection_randoms
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _ws(nbytes: int) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=DEV)


def test_empty_set_every_entry_point():
    hm = mesh()
    dm = DeviceMesh(hm, DEV, mixed=False, dist=hm.inject_distribution(200))
    dmx = DeviceMesh(hm, DEV, mixed=True)
    lib = L.load()
    ps = ParticleSet(DEV, 64)
    ps.size = 0
    ps.status.fill_(-1)  # every move entry point must reset it
    v = ps.view()
    charge = torch.zeros(hm.n_nodes, dtype=torch.float64, device=DEV)
    dws = _ws(lib.oppb_deposit_workspace_bytes(hm.n_nodes))
    st = ps.status.data_ptr()
    calls = {
        "move_f64": lambda: lib.oppb_move_f64(C.byref(dm.s), C.byref(v), st, 64, None),
        "move_deposit_f64": lambda: lib.oppb_move_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(), st, 64,
                                                              dws.data_ptr(), dws.numel(), None),
        "move_deposit_mixed": lambda: lib.oppb_move_deposit_mixed(C.byref(dmx.s), C.byref(v), charge.data_ptr(), st,
                                                                  64, 1e-5, dws.data_ptr(), dws.numel(), None),
        "push_move_deposit_mixed": lambda: lib.oppb_push_move_deposit_mixed(
            C.byref(dmx.s), C.byref(v), charge.data_ptr(), st, 64, 1e-5, 1.0, 0.01, dws.data_ptr(), dws.numel(), None),
        "push_f64": lambda: lib.oppb_push_f64(C.byref(dm.s), C.byref(v), 1.0, 0.01, None),
        "deposit_f64": lambda: lib.oppb_deposit_f64(C.byref(dm.s), C.byref(v), charge.data_ptr(), dws.data_ptr(),
                                                    dws.numel(), None),
    }
    for name, call in calls.items():
        ps.status.fill_(-1)
        assert call() == L.OPPB_OK, name
        torch.cuda.synchronize()
        if name.startswith(("move", "push_move")):
            s = ps.status_host()
            assert (s.remove_count, int(s.total_visits), s.error) == (0, 0, 0), name
    assert not charge.any()
    rd = randoms_to_device(injection_randoms(0, 0, 200, 0.1), DEV)
    assert lib.oppb_inject_f64(C.byref(dm.s), C.byref(dm.inlet), C.byref(v), 0, 0, rd.data_ptr(), rd.stride(0), 5,
                               1.0, 1.0, 0.01, None) == L.OPPB_OK
    dats = ps.dat_list()
    hws = _ws(lib.oppb_hole_fill_workspace_bytes(0, 0))
    assert lib.oppb_hole_fill(0, 0, ps.bits.data_ptr(), ps.capacity, 4, dats, hws.data_ptr(), hws.numel(),
                              None) == L.OPPB_OK
    sws = _ws(lib.oppb_sort_workspace_bytes(0, hm.n_cells))
    assert lib.oppb_sort_by_cell(0, hm.n_cells, ps.capacity, 4, dats, 3, None, sws.data_ptr(), sws.numel(),
                                 None) == L.OPPB_OK
    torch.cuda.synchronize()


def _sorted_state(n, n_cells, frac_removed, seed):
    rng = np.random.default_rng(seed)
    pos, vel, lc = rng.random((n, 3)), rng.random((n, 3)), rng.random((n, 4))
    p2c = rng.integers(0, n_cells, n).astype(np.int32)
    p2c[rng.random(n) < frac_removed] = REMOVED
    return pos, vel, lc, p2c


def _load(ps, pos, vel, lc, p2c):
    n = len(p2c)
    ps.size = n
    ps.pos[:, :n] = torch.from_numpy(pos.T.copy()).to(DEV)
    ps.vel[:, :n] = torch.from_numpy(vel.T.copy()).to(DEV)
    ps.lc[:, :n] = torch.from_numpy(lc.T.copy()).to(DEV)
    ps.p2c[0, :n] = torch.from_numpy(p2c).to(DEV)


@pytest.mark.parametrize("n,n_cells,frac", [(200_003, (1 << 24) + 5, 0.05),   # 25 key bits: four passes
                                            (70_001, 1, 0.3),                  # one key bit, one pass
                                            (4099, (1 << 30) + 7, 0.0)])       # 31 key bits
def test_sort_key_widths(n, n_cells, frac):
    pos, vel, lc, p2c = _sorted_state(n, n_cells, frac, 11)
    ps = ParticleSet(DEV, n)
    _load(ps, pos, vel, lc, p2c)
    lib = L.load()
    ws = _ws(lib.oppb_sort_workspace_bytes(n, n_cells))
    perm = torch.empty(n, dtype=torch.int32, device=DEV)
    L.check("sort", lib.oppb_sort_by_cell(n, n_cells, ps.capacity, 4, ps.dat_list(), 3, perm.data_ptr(),
                                          ws.data_ptr(), ws.numel(), None))
    ps.swap_after_sort()
    # The order: stable by cell, removed particles last.  The oracle's counting sort holds an
    # array of n_cells counters, so the 31-bit case is checked with numpy's stable sort of the
    # same keys (the two agree wherever both run).
    keys = np.where(p2c == REMOVED, np.int64(n_cells), p2c.astype(np.int64))
    perm_np = np.argsort(keys, kind="stable").astype(np.int32)
    dats = [pos.copy(), vel.copy(), lc.copy(), p2c.copy()]
    if n_cells <= (1 << 25):
        perm_o = O.sort(n, n_cells, dats, 3)
        np.testing.assert_array_equal(perm_o, perm_np)
    else:
        dats = [d[perm_np] for d in dats]
    np.testing.assert_array_equal(perm.cpu().numpy(), perm_np)
    got = ps.host_aos()
    for k, name in enumerate(("pos", "vel", "lc", "p2c")):
        np.testing.assert_array_equal(got[name].view(np.uint8), dats[k].view(np.uint8), err_msg=name)


@pytest.mark.parametrize("where", ["tail", "head"])
def test_hole_fill_holes_at_one_end(where):
    n, r = 50_000, 3_000
    pos, vel, lc, p2c = _sorted_state(n, 24000, 0.0, 5)
    if where == "tail":
        p2c[n - r:] = REMOVED   # nothing to move: the live prefix is already contiguous
    else:
        p2c[:r] = REMOVED       # every hole is filled from the tail
    ps = ParticleSet(DEV, n)
    _load(ps, pos, vel, lc, p2c)
    bits = np.packbits((p2c == REMOVED).astype(np.uint8), bitorder="little")
    words = np.zeros(ps.bits.numel() * 4, np.uint8)
    words[: len(bits)] = bits
    ps.bits.copy_(torch.from_numpy(words.view(np.int32)).to(DEV))
    lib = L.load()
    ws = _ws(lib.oppb_hole_fill_workspace_bytes(n, r))
    L.check("hole_fill", lib.oppb_hole_fill(n, r, ps.bits.data_ptr(), ps.capacity, 4, ps.dat_list(), ws.data_ptr(),
                                            ws.numel(), None))
    dats = [pos.copy(), vel.copy(), lc.copy(), p2c.copy()]
    O.hole_fill(n, r, dats[3], dats)
    got = ps.host_aos()
    for k, name in enumerate(("pos", "vel", "lc", "p2c")):
        np.testing.assert_array_equal(got[name][: n - r].view(np.uint8), dats[k][: n - r].view(np.uint8),
                                      err_msg=name)


def test_hole_fill_many_bitmap_blocks():
    """A hole fill over 70M particles: more bitmap blocks (4,273 of 16,384 particles) than the
    single-block scan takes in one 4,096-value pass, so the block counts are scanned in two
    passes.  Two int32 dats (the cells and each particle's index) against the pairing rule:
    the k-th hole in ascending order takes the k-th live particle from the back while that one
    lies behind it."""
    n, r = 70_000_003, 7_001
    rng = np.random.default_rng(21)
    holes = np.sort(rng.choice(n, r, replace=False))
    p2c = (np.arange(n, dtype=np.int64) % 1000).astype(np.int32)
    p2c[holes] = REMOVED
    ident = np.arange(n, dtype=np.int32)
    bits = np.packbits((p2c == REMOVED).astype(np.uint8), bitorder="little")
    words = np.zeros((n + 31) // 32 * 4, np.uint8)
    words[: len(bits)] = bits
    d_p2c, d_ident = torch.from_numpy(p2c).to(DEV), torch.from_numpy(ident).to(DEV)
    d_bits = torch.from_numpy(words.view(np.int32)).to(DEV)
    dats = (L.Dat * 2)(L.Dat(d_p2c.data_ptr(), None, 1, 4), L.Dat(d_ident.data_ptr(), None, 1, 4))
    lib = L.load()
    ws = _ws(lib.oppb_hole_fill_workspace_bytes(n, r))
    L.check("hole_fill", lib.oppb_hole_fill(n, r, d_bits.data_ptr(), n, 2, dats, ws.data_ptr(), ws.numel(), None))
    got_p2c, got_ident = d_p2c.cpu().numpy(), d_ident.cpu().numpy()
    live_back = np.flatnonzero(p2c != REMOVED)[::-1][:r]
    keep = live_back > holes
    want_p2c, want_ident = p2c.copy(), ident.copy()
    want_p2c[holes[keep]] = p2c[live_back[keep]]
    want_ident[holes[keep]] = ident[live_back[keep]]
    np.testing.assert_array_equal(got_p2c[: n - r], want_p2c[: n - r])
    np.testing.assert_array_equal(got_ident[: n - r], want_ident[: n - r])
    assert not (got_p2c[: n - r] == REMOVED).any()
