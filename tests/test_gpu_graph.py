"""Whole FemPIC steps captured as one CUDA graph (include/oppb_graph.h) and the shuffle fill
modes.

A graph replay runs S steps (node charge reset, inject, push + move + deposit, hole fill / cell
sort / shuffle, step record) with the particle count in device memory and reads the count and
the records back once.  It must give what S direct steps (FemPIC.step, which reads the remove
count after every move as the reference's opp_finalize_particle_move does) give on the same
tables: the same per-step counts and visits, the same particle dats bit for bit, node charges
within 1e-12 (FP64 atomics add in a run-dependent order), and the oracle's results.

The shuffles (opp_fill = Shuffle_All / Shuffle_Periodic) order the live particles by random
keys, so the order is not the reference's (its keys come from Thrust's engine); the particles
themselves must be those of the seq backend, whose shuffle sorts by cell
(opp_lib/src/core/opp_particle_organize_core.cpp:98-121): the same rows as the oracle's sorted
run, step for step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from helpers import mesh
from oppb import _lib as L
from oppb.fempic import FemPIC, injection_randoms, randoms_to_device
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
CHARGE_RTOL = 1e-12
INJECT = 2000


def _tables(seed: int, first: int, count: int):
    return [randoms_to_device(injection_randoms(seed, first + k, INJECT, 0.1), DEV) for k in range(count)]


def _charge_close(a: np.ndarray, b: np.ndarray, rtol: float = CHARGE_RTOL) -> None:
    err = np.abs(a - b) / np.maximum(np.abs(b), 1.0)
    assert err.max() <= rtol, f"node charge max rel err {err.max():.3e}"


def _same_dats(a: FemPIC, b: FemPIC) -> None:
    ga, gb = a.parts.host_aos(), b.parts.host_aos()
    for name in ("p2c", "pos", "vel", "lc"):
        np.testing.assert_array_equal(ga[name].view(np.uint8), gb[name].view(np.uint8), err_msg=name)


def _rows(p2c, pos, vel, lc) -> np.ndarray:
    """Particle rows as bytes, sorted: the multiset of particles whatever their order."""
    rec = np.concatenate([p2c.astype(np.int64)[:, None].view(np.uint64), pos.view(np.uint64), vel.view(np.uint64),
                          lc.view(np.uint64)], axis=1)
    return rec[np.lexsort(rec.T[::-1])]


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("fill", ["HoleFill_All", "Sort_Periodic", "Sort_All", "Shuffle_Periodic"])
def test_graph_replays_equal_direct_steps(precision, fill):
    """60 steps as 6 replays of a 10-step graph against 60 direct steps, same tables."""
    hm = mesh()
    kw = dict(inject_per_step=INJECT, precision=precision, fill=fill, fill_period=5)
    direct, graphed = FemPIC(hm, DEV, **kw), FemPIC(hm, DEV, **kw)
    S, removed = 10, 0
    for r in range(6):
        tabs = _tables(3, r * S, S)
        want = [direct.step(t) for t in tabs]
        got = graphed.run_graph(tabs)
        for k, (a, b) in enumerate(zip(want, got)):
            key = ("size_before_move", "removed", "size", "visits", "max_visits", "rechecks")
            assert tuple(a[x] for x in key) == tuple(b[x] for x in key), (r, k)
            removed += a["removed"]
        assert graphed.parts.size == direct.parts.size and graphed.iter == direct.iter
    _same_dats(direct, graphed)
    _charge_close(graphed.node_charge.cpu().numpy(), direct.node_charge.cpu().numpy())
    assert removed > 0 and direct.parts.size > 50_000


@pytest.mark.parametrize("fill", ["Sort_All", "Shuffle_All"])
def test_graph_sort_without_removals_copies(fill):
    """Without thermal spread no ion leaves the box in the first steps: every step's sort (or
    shuffle) finds nothing removed, the reference does nothing, and the graph's sort copies the
    dats into their swap buffers unchanged; the state equals the direct steps' bit for bit."""
    hm = mesh()
    kw = dict(inject_per_step=INJECT, fill=fill)
    direct, graphed = FemPIC(hm, DEV, **kw), FemPIC(hm, DEV, **kw)
    for r in range(3):
        tabs = [randoms_to_device(injection_randoms(4, r * 5 + k, INJECT, 0.0), DEV) for k in range(5)]
        want = [direct.step(t) for t in tabs]
        got = graphed.run_graph(tabs)
        assert all(a["removed"] == 0 and a["compaction"] == "none" for a in want)
        assert [b["size"] for b in got] == [a["size"] for a in want]
    _same_dats(direct, graphed)


def test_graph_steps_match_oracle():
    """Graph replays against the C oracle (bit-exact state, per-step counts and visits)."""
    hm = mesh()
    sim = FemPIC(hm, DEV, inject_per_step=INJECT, fill="Sort_Periodic", fill_period=10)
    orc = O.OracleFemPIC(hm, sim.dist_host, fill="Sort_Periodic", fill_period=10)
    S = 10
    for r in range(5):
        rnds = [injection_randoms(7, r * S + k, INJECT, 0.1) for k in range(S)]
        got = sim.run_graph([randoms_to_device(x, DEV) for x in rnds])
        for k, x in enumerate(rnds):
            o = orc.step(x)
            assert (got[k]["size_before_move"], got[k]["removed"], got[k]["size"], got[k]["visits"]) == \
                (o["size_before_move"], o["removed"], o["size"], o["visits"]), (r, k)
    g, n = sim.parts.host_aos(), orc.size
    np.testing.assert_array_equal(g["p2c"], orc.p2c[:n])
    for name in ("pos", "vel", "lc"):
        np.testing.assert_array_equal(g[name].view(np.uint64), getattr(orc, name)[:n].view(np.uint64), err_msg=name)
    _charge_close(sim.node_charge.cpu().numpy(), orc.node_charge)


def test_graph_is_reused_and_recaptured():
    """A replay reuses the captured graph while the count stays within its bound; growth past
    the bound captures again (and results stay those of direct steps)."""
    hm = mesh()
    direct = FemPIC(hm, DEV, inject_per_step=INJECT, fill="HoleFill_All")
    graphed = FemPIC(hm, DEV, inject_per_step=INJECT, fill="HoleFill_All")
    S = 4
    seen = set()
    for r in range(8):
        tabs = _tables(5, r * S, S)
        for t in tabs:
            direct.step(t)
        g = graphed.graph_for(S)
        seen.add(id(g))
        for dst, src in zip(g.tables, tabs):
            dst.copy_(src)
        graphed.replay(g)
        assert graphed.parts.size == direct.parts.size
    assert 1 < len(seen) <= 8  # growing count: new bounds
    # With a count that stays put (no injection growth beyond the slack) the graph is reused.
    g1 = graphed.graph_for(S)
    assert graphed.graph_for(S) is g1
    _same_dats(direct, graphed)


def test_inject_dev_refuses_overflow():
    """oppb_inject_dev with a device count too close to the capacity writes nothing and
    records OPPB_ERR_CAPACITY."""
    hm = mesh()
    sim = FemPIC(hm, DEV, inject_per_step=100, capacity=1000)
    p = sim.parts
    p.p2c.fill_(L.REMOVED_CELL)
    before = p.p2c.clone()
    count = torch.tensor([p.capacity - 10, 0, 0, 0], dtype=torch.int32, device=DEV)
    tab = randoms_to_device(injection_randoms(1, 0, 100, 0.1), DEV)
    v = p.view()
    L.check("oppb_inject_dev", sim.lib.oppb_inject_dev(
        C.byref(sim.mesh.s), C.byref(sim.mesh.inlet), C.byref(v), count.data_ptr(), 100, tab.data_ptr(),
        tab.stride(0), 5, 1.0, 1.0, 0.01, None))
    torch.cuda.synchronize()
    assert int(count[1]) == L.OPPB_ERR_CAPACITY and int(count[0]) == p.capacity - 10
    assert torch.equal(p.p2c, before)


@pytest.mark.parametrize("fill", ["Shuffle_All", "Shuffle_Periodic"])
def test_shuffle_fill_modes_hold_the_oracles_particles(fill):
    """After every step the particles (cells, positions, velocities, weights) are those of the
    oracle running the seq backend's shuffle (a sort by cell), in another order."""
    hm = mesh()
    sim = FemPIC(hm, DEV, inject_per_step=INJECT, fill=fill, fill_period=4)
    orc = O.OracleFemPIC(hm, sim.dist_host, fill=fill.replace("Shuffle", "Sort"), fill_period=4)
    shuffled_unsorted = 0
    for s in range(40):
        rnd = injection_randoms(9, s, INJECT, 0.1)
        g = sim.step(randoms_to_device(rnd, DEV))
        o = orc.step(rnd)
        assert (g["size_before_move"], g["removed"], g["size"], g["visits"]) == \
            (o["size_before_move"], o["removed"], o["size"], o["visits"]), s
        if s % 4 == 0 or s == 39:
            got, n = sim.parts.host_aos(), orc.size
            np.testing.assert_array_equal(_rows(got["p2c"], got["pos"], got["vel"], got["lc"]),
                                          _rows(orc.p2c[:n], orc.pos[:n], orc.vel[:n], orc.lc[:n]), err_msg=str(s))
            if g["compaction"] == "shuffle" and np.any(np.diff(got["p2c"]) < 0):
                shuffled_unsorted += 1
        _charge_close(sim.node_charge.cpu().numpy(), orc.node_charge)
    assert shuffled_unsorted > 0 and orc.size > 50_000


def test_shuffle_removed_last_and_permutation():
    """oppb_shuffle: a stable order of random keys, removed particles last, the permutation
    covering every index once, and the same seed giving the same order."""
    from oppb.fempic import ParticleSet

    n, n_cells = 100_003, 5000
    rng = np.random.default_rng(4)
    p2c = rng.integers(0, n_cells, n).astype(np.int32)
    p2c[rng.random(n) < 0.05] = L.REMOVED_CELL
    perms = []
    for _ in range(2):
        ps = ParticleSet(DEV, n)
        ps.size = n
        ps.p2c[0, :n] = torch.from_numpy(p2c).to(DEV)
        ps.pos[0, :n] = torch.arange(n, dtype=torch.float64, device=DEV)
        nb = L.load().oppb_sort_workspace_bytes(n, n_cells)
        ws = torch.empty(nb, dtype=torch.uint8, device=DEV)
        perm = torch.empty(n, dtype=torch.int32, device=DEV)
        L.check("oppb_shuffle", L.load().oppb_shuffle(n, n_cells, ps.capacity, len(ps.DATS), ps.dat_list(), 3,
                                                      0x1234, perm.data_ptr(), ws.data_ptr(), nb, None))
        ps.swap_after_sort()
        got = ps.host_aos()
        pm = perm.cpu().numpy()
        assert np.array_equal(np.sort(pm), np.arange(n))
        np.testing.assert_array_equal(got["p2c"], p2c[pm])
        np.testing.assert_array_equal(got["pos"][:, 0], pm.astype(np.float64))
        live = int((p2c != L.REMOVED_CELL).sum())
        assert np.all(got["p2c"][live:] == L.REMOVED_CELL) and np.all(got["p2c"][:live] != L.REMOVED_CELL)
        assert np.any(np.diff(pm[:live]) < 0)  # not the identity: shuffled
        perms.append(pm)
    np.testing.assert_array_equal(perms[0], perms[1])


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_run_graph_host_equals_run_steps(precision):
    """FemPIC.run_graph_host (graph replays of 10 steps, staging copies on a second stream, every
    step's node charges copied aside inside the graph) against FemPIC.run_steps on the same
    pinned host tables: 25 steps (chunks of 10, 10 and 5), the same per-step counts and visits,
    the same particle dats bit for bit, every step's node charges within 1e-12; then a second
    call that replays the graphs it captured."""
    hm = mesh()
    kw = dict(inject_per_step=INJECT, precision=precision, fill="Sort_Periodic", fill_period=10)
    a, b = FemPIC(hm, DEV, **kw), FemPIC(hm, DEV, **kw)
    n = 25
    host = [torch.from_numpy(np.ascontiguousarray(injection_randoms(6, k, INJECT, 0.1).T)).pin_memory()
            for k in range(2 * n)]
    ca = [torch.empty(hm.n_nodes, dtype=torch.float64).pin_memory() for _ in range(2 * n)]
    cb = [torch.empty(hm.n_nodes, dtype=torch.float64).pin_memory() for _ in range(2 * n)]
    key = ("size_before_move", "removed", "size", "visits", "max_visits", "rechecks")
    for half in range(2):
        sl = slice(half * n, (half + 1) * n)
        ra = a.run_steps(host[sl], ca[sl])
        graphs_before = len(b._graphs)
        rb = b.run_graph_host(host[sl], cb[sl])
        assert [tuple(x[k] for k in key) for x in ra] == [tuple(x[k] for k in key) for x in rb], half
        for k in range(sl.start, sl.stop):
            _charge_close(cb[k].numpy(), ca[k].numpy())
        _charge_close(b.node_charge.cpu().numpy(), ca[sl.stop - 1].numpy())
        _same_dats(a, b)
        assert a.iter == b.iter and a.parts.size == b.parts.size
    assert len(b._graphs) >= graphs_before  # the second call reuses or adds graphs, never fewer
    assert b.parts.size > 40_000


def test_run_graph_host_rejects_mixed_counts():
    hm = mesh()
    sim = FemPIC(hm, DEV, inject_per_step=INJECT)
    t = [torch.zeros((5, INJECT), dtype=torch.float64).pin_memory(),
         torch.zeros((5, INJECT + 1), dtype=torch.float64).pin_memory()]
    with pytest.raises(ValueError):
        sim.run_graph_host(t)
