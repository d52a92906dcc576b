"""oppb_hole_fill_static: the hole fill for callers that cannot allocate device memory
where they compact particles (a plugin that only holds the dats' device pointers while
another runtime owns the memory, or a step loop that cannot pay the device-wide
synchronisation of cudaMalloc / cudaFree).  Its scratch is a fixed array inside the
library, so it takes no workspace.

Checked against oppb_hole_fill (the workspace entry point) on the same inputs, bit for
bit like every hole-fill test, over two calls in a row: the second call is smaller than
the first, so a result that depended on scratch contents left by the first call would
show.  This file is named to be collected last."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oppb import _lib as L
from oppb.fempic import ParticleSet

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REMOVED = L.REMOVED_CELL


def _loaded_set(pos, vel, lc, p2c) -> ParticleSet:
    n = len(p2c)
    ps = ParticleSet(DEV, n)
    ps.increase(n)
    ps.size = n
    ps.pos[:, :n] = torch.from_numpy(pos.T.copy()).to(DEV)
    ps.vel[:, :n] = torch.from_numpy(vel.T.copy()).to(DEV)
    ps.lc[:, :n] = torch.from_numpy(lc.T.copy()).to(DEV)
    ps.p2c[0, :n] = torch.from_numpy(p2c).to(DEV)
    bits = np.packbits((p2c == REMOVED).astype(np.uint8), bitorder="little")
    words = np.zeros(ps.bits.numel() * 4, np.uint8)
    words[: len(bits)] = bits
    ps.bits.copy_(torch.from_numpy(words.view(np.int32)).to(DEV))
    return ps


def _state(n, frac, seed):
    rng = np.random.default_rng(seed)
    p2c = rng.integers(0, 2_654_208, n).astype(np.int32)
    p2c[rng.random(n) < frac] = REMOVED
    return rng.random((n, 3)), rng.random((n, 3)), rng.random((n, 4)), p2c


def _with_workspace(state) -> dict:
    ps = _loaded_set(*state)
    n, R = ps.size, int((state[3] == REMOVED).sum())
    lib = L.load()
    nb = lib.oppb_hole_fill_workspace_bytes(n, R)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=DEV)
    L.check("oppb_hole_fill", lib.oppb_hole_fill(n, R, ps.bits.data_ptr(), ps.capacity, 4, ps.dat_list(),
                                                 ws.data_ptr(), nb, None))
    torch.cuda.synchronize()
    return ps.host_aos()


def _static(state) -> dict:
    ps = _loaded_set(*state)
    n, R = ps.size, int((state[3] == REMOVED).sum())
    L.check("oppb_hole_fill_static", L.load().oppb_hole_fill_static(n, R, ps.bits.data_ptr(), ps.capacity, 4,
                                                                    ps.dat_list(), None))
    torch.cuda.synchronize()
    return ps.host_aos()


def test_static_hole_fill_matches_workspace_entry_point_twice():
    # First call: 1,000,003 particles with about 200k removals; second call: fewer
    # particles and removals, in the part of the scratch the first call left filled.
    for n, frac, seed in ((1_000_003, 0.2, 11), (70_001, 0.05, 12)):
        state = _state(n, frac, seed)
        R = int((state[3] == REMOVED).sum())
        assert 0 < R <= L.HOLE_FILL_STATIC_MAX_REMOVES
        want = _with_workspace(state)
        got = _static(state)
        for name in ("pos", "vel", "lc", "p2c"):
            np.testing.assert_array_equal(got[name][: n - R].view(np.uint8), want[name][: n - R].view(np.uint8),
                                          err_msg=f"{name} (n={n}, removed={R})")
        assert not (got["p2c"][: n - R] == REMOVED).any()


def test_static_hole_fill_rejects_more_removals_than_its_scratch_holds():
    state = _state(1000, 0.1, 13)
    ps = _loaded_set(*state)
    before = ps.host_aos()
    rc = L.load().oppb_hole_fill_static(ps.size, L.HOLE_FILL_STATIC_MAX_REMOVES + 1, ps.bits.data_ptr(),
                                        ps.capacity, 4, ps.dat_list(), None)
    assert rc == L.OPPB_ERR_SCRATCH_LIMIT
    assert b"scratch" in L.load().oppb_status_string(rc)
    torch.cuda.synchronize()
    after = ps.host_aos()
    for name in before:
        np.testing.assert_array_equal(after[name], before[name])
