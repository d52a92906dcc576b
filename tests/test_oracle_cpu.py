"""The C oracle against the reference: the golden fixtures (made by the compiled
reference seq backend, tests/golden/make_golden.py) always, and the live compiled
reference on the 10x10x40-hex case when oracle/_ref is built."""
from __future__ import annotations

from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_runner as R

GOLDEN = Path(__file__).resolve().parent / "golden"


def _golden(name):
    z = np.load(GOLDEN / f"{name}.npz")
    mesh = SimpleNamespace(**{k: z[k] for k in ("c2n", "c2c", "c_det", "c_vol", "c_ef", "if2c", "if_u", "if_v",
                                                "if_norm", "if_n_pos")})
    mesh.n_nodes, mesh.n_cells, mesh.n_ifaces = int(z["n_nodes"]), int(z["n_cells"]), int(z["n_ifaces"])
    if "n_pos" in z:
        mesh.n_pos = z["n_pos"]
    return z, mesh


@pytest.mark.parametrize("name", ["fempic_4x4x8_holefill", "fempic_4x4x8_sort"])
def test_oracle_matches_golden(name):
    z, mesh = _golden(name)
    o = O.OracleFemPIC(mesh, z["dist"], fill=str(z["fill"]), fill_period=int(z["period"]))
    recs = z["records"]
    for s in range(int(z["steps"])):
        r = o.step(z["tables"][s])
        rec = recs[s]
        n = o.size
        assert (r["size"], r["removed"]) == (int(rec["size"]), int(rec["removed"])), s
        assert R.fnv1a(o.p2c[:n]) == int(rec["h_p2c"]), s
        assert R.fnv1a(o.pos[:n]) == int(rec["h_pos"]), s
        assert R.fnv1a(o.vel[:n]) == int(rec["h_vel"]), s
        assert R.fnv1a(o.lc[:n]) == int(rec["h_lc"]), s
        assert R.fnv1a(o.node_charge) == int(rec["h_charge"]), s
    n = o.size
    np.testing.assert_array_equal(o.p2c[:n], z["p2c"])
    np.testing.assert_array_equal(o.pos[:n].view(np.uint64), z["pos"].view(np.uint64))
    np.testing.assert_array_equal(o.lc[:n].view(np.uint64), z["lc"].view(np.uint64))
    np.testing.assert_array_equal(o.node_charge.view(np.uint64), z["node_charge"].view(np.uint64))
    # golden cases exercise removals, and the sort case sorts
    assert recs["removed"].sum() > 0


def test_golden_invariants():
    """Properties the reference's state obeys: charge sum = particle count (weights sum
    to 1), every live particle's weights lie in the inside band of its cell."""
    z, mesh = _golden("fempic_4x4x8_sort")
    n = len(z["p2c"])
    assert abs(z["node_charge"].sum() - n) < 1e-9 * n
    assert (z["lc"] > -1e-10).all() and (z["lc"] - 1.0 < 1e-10).all()
    assert ((z["p2c"] >= 0) & (z["p2c"] < mesh.n_cells)).all()


@pytest.mark.skipif(not R.available("seq_stable"), reason="compiled reference not built (needs its sources)")
@pytest.mark.parametrize("fill,steps,period", [("HoleFill_All", 120, 10), ("Sort_Periodic", 60, 5)])
def test_oracle_matches_live_reference(fill, steps, period):
    from helpers import mesh as mk
    from oppb.fempic import injection_randoms

    hm = mk()
    dist = hm.inject_distribution(2000)
    tables = [injection_randoms(5, s, 2000, 0.1) for s in range(steps)]
    ref = R.run("seq_stable", hm, dist, steps, tables, fill=fill, period=period)
    o = O.OracleFemPIC(hm, dist, fill=fill, fill_period=period)
    for s in range(steps):
        o.step(tables[s])
        rec = ref["records"][s]
        n = o.size
        assert o.size == rec["size"]
        assert R.fnv1a(o.p2c[:n]) == int(rec["h_p2c"]), s
        assert R.fnv1a(o.lc[:n]) == int(rec["h_lc"]), s
        assert R.fnv1a(o.node_charge) == int(rec["h_charge"]), s


@pytest.mark.skipif(not R.available("seq"), reason="compiled reference not built (needs its sources)")
def test_stock_seq_sort_differs_only_within_cells():
    """The shipped seq backend sorts with std::sort (unstable): same cells per position
    after a sort, possibly a different particle order inside a cell."""
    from helpers import mesh as mk
    from oppb.fempic import injection_randoms

    hm = mk()
    dist = hm.inject_distribution(2000)
    tables = [injection_randoms(6, s, 2000, 0.1) for s in range(21)]
    a = R.run("seq_stable", hm, dist, 21, tables, fill="Sort_Periodic", period=10)
    b = R.run("seq", hm, dist, 21, tables, fill="Sort_Periodic", period=10)
    assert a["size"] == b["size"]
    np.testing.assert_array_equal(np.sort(a["p2c"]), np.sort(b["p2c"]))
    np.testing.assert_array_equal(np.sort(a["node_charge"]), np.sort(a["node_charge"]))


def test_hole_fill_pairs_follow_reference_rule():
    """k-th hole (ascending) takes the k-th live particle from the back while it lies behind."""
    rng = np.random.default_rng(0)
    for trial in range(50):
        n = int(rng.integers(1, 300))
        p2c = rng.integers(0, 10, n).astype(np.int32)
        rem = rng.random(n) < rng.random()
        p2c[rem] = O.REMOVED
        R_ = int(rem.sum())
        data = np.arange(n, dtype=np.float64).reshape(n, 1).copy()
        p = p2c.copy()
        pf, pt = O.hole_fill(n, R_, p, [data, p])
        holes = np.flatnonzero(p2c == O.REMOVED)
        live_back = np.flatnonzero(p2c != O.REMOVED)[::-1]
        k = 0
        while k < min(R_, len(holes), len(live_back)) and live_back[k] > holes[k]:
            k += 1
        np.testing.assert_array_equal(pt, holes[:k])
        np.testing.assert_array_equal(pf, live_back[:k])
        assert not (p[: n - R_] == O.REMOVED).any()


def test_oracle_sort_is_stable():
    rng = np.random.default_rng(1)
    n = 5000
    p2c = rng.integers(0, 50, n).astype(np.int32)
    p2c[rng.random(n) < 0.1] = O.REMOVED
    idx = np.arange(n, dtype=np.float64).reshape(n, 1).copy()
    key = p2c.copy()
    perm = O.sort(n, 50, [idx, key], 1)
    ref = np.argsort(np.where(p2c == O.REMOVED, 50, p2c), kind="stable")
    np.testing.assert_array_equal(perm, ref)
    np.testing.assert_array_equal(idx[:, 0], ref.astype(np.float64))


def test_dh_oracle_matches_golden():
    """Direct hop: the structured grid (box counts, bounds, every map entry) and 30 global-move
    steps of the reference seq backend (fixture made by tests/golden/make_golden.py)."""
    z, mesh = _golden("fempic_4x4x8_dh")
    sp = float(z["spacing"])
    dh = O.DirectHop(z["n_pos"], sp, (4 * sp,) * 3, mesh=mesh)
    np.testing.assert_array_equal(dh.dims, z["dh_dims"])
    np.testing.assert_array_equal(dh.box.view(np.uint64), z["dh_box"].view(np.uint64))
    np.testing.assert_array_equal(dh.map, z["dh_map"])
    assert 0 < (dh.map != O.REMOVED).sum() < dh.size  # boxes inside and outside the mesh
    o = O.OracleFemPIC(mesh, z["dist"], dt=float(z["dt"]), fill=str(z["fill"]), fill_period=int(z["period"]), dh=dh)
    for s in range(int(z["steps"])):
        r = o.step(z["tables"][s])
        rec = z["records"][s]
        n = o.size
        assert (r["size"], r["removed"]) == (int(rec["size"]), int(rec["removed"])), s
        assert R.fnv1a(o.p2c[:n]) == int(rec["h_p2c"]), s
        assert R.fnv1a(o.pos[:n]) == int(rec["h_pos"]), s
        assert R.fnv1a(o.lc[:n]) == int(rec["h_lc"]), s
        assert R.fnv1a(o.node_charge) == int(rec["h_charge"]), s
    np.testing.assert_array_equal(o.p2c[:o.size], z["p2c"])


def test_dh_seed_removes_outside_grid():
    """Positions outside the grid, or in a box without a cell, are removed (the CUDA
    backend's rule); inside, p2c becomes the box's cell."""
    z, mesh = _golden("fempic_4x4x8_dh")
    sp = float(z["spacing"])
    dh = O.DirectHop(z["n_pos"], sp, (4 * sp,) * 3)
    dh.map = z["dh_map"].copy()
    lo, hi = dh.box[:3], dh.box[3:]
    pos = np.array([[0.5, 0.5, 1.0],            # inside the mesh
                    [lo[0] - 1.0, 0.5, 1.0],    # below the grid in x
                    [0.5, hi[1] + 1.0, 1.0],    # above the grid in y
                    [-0.3, -0.3, -0.3],         # in the grid, outside the mesh (no cell)
                    [np.nan, 0.5, 1.0]])        # NaN truncates to box 0: no cell there
    p2c = np.zeros(len(pos), np.int32)
    assert dh.seed(pos, p2c) == 4
    assert p2c[0] != O.REMOVED and (p2c[1:] == O.REMOVED).all()
    ix = ((pos[0] - lo) * dh.inv).astype(np.int64)
    assert p2c[0] == dh.map[ix[0] + dh.dims[0] * (ix[1] + dh.dims[1] * ix[2])]


@pytest.mark.skipif(not R.available("seq_stable"), reason="compiled reference not built (needs its sources)")
def test_dh_oracle_matches_live_reference():
    """A spacing that does not divide the box and unequal expansions (the reference widens
    both x and y minima by the x expansion and both maxima by the y expansion)."""
    from oppb.fempic import HostMesh, injection_randoms

    hm = HostMesh(5, 3, 6, 1.0, 0.6, 1.2)
    dist = hm.inject_distribution(150)
    steps = 20
    tables = [injection_randoms(9, s, 150, 0.1) for s in range(steps)]
    sp, ex = 0.07, (0.3, 0.2, 0.25)
    ref = R.run("seq_stable", hm, dist, steps, tables, fill="HoleFill_All", period=10, dt=0.2, dh=(sp, ex))
    dh = O.DirectHop(hm.n_pos, sp, ex, mesh=hm)
    np.testing.assert_array_equal(dh.dims, ref["dh_dims"])
    np.testing.assert_array_equal(dh.box.view(np.uint64), ref["dh_box"].view(np.uint64))
    np.testing.assert_array_equal(dh.map, ref["dh_map"])
    o = O.OracleFemPIC(hm, dist, dt=0.2, fill="HoleFill_All", fill_period=10, dh=dh)
    for s in range(steps):
        o.step(tables[s])
        rec = ref["records"][s]
        n = o.size
        assert o.size == rec["size"], s
        assert R.fnv1a(o.p2c[:n]) == int(rec["h_p2c"]), s
        assert R.fnv1a(o.lc[:n]) == int(rec["h_lc"]), s
        assert R.fnv1a(o.node_charge) == int(rec["h_charge"]), s


def test_oracle_deposit_exact_definition():
    """deposit_exact against exact rational arithmetic on a small case: per node, the sum of
    floor(w 2^52) 2^-52 over its particles' weights, rounded once to FP64; removed particles
    skipped; and within a few FP64 rounding units of the oracle's sequential deposit."""
    from fractions import Fraction

    rng = np.random.default_rng(4)
    n_cells, n_nodes, n = 40, 30, 500
    c2n = np.stack([rng.choice(n_nodes, 4, replace=False) for _ in range(n_cells)]).astype(np.int32)
    p2c = rng.integers(0, n_cells, n).astype(np.int32)
    p2c[::17] = O.REMOVED
    lc = rng.uniform(-1e-10, 1.0, (n, 4))
    lc[3] = [-2.0 ** -52 * 1.5, 2.0 ** -60, 0.3, 1.0]
    got = O.deposit_exact(lc, p2c, c2n, n_nodes)
    ref = [Fraction(0)] * n_nodes
    for i in range(n):
        if p2c[i] == O.REMOVED:
            continue
        for k in range(4):
            ref[c2n[p2c[i], k]] += Fraction(int(np.floor(lc[i, k] * 2.0 ** 52)), 2 ** 52)
    np.testing.assert_array_equal(got, np.array([float(r) for r in ref]))  # float(Fraction) rounds once
    keep = p2c != O.REMOVED
    seq = np.zeros(n_nodes)
    O.deposit(np.ascontiguousarray(lc[keep]), np.ascontiguousarray(p2c[keep]), c2n, seq)
    assert np.abs(got - seq).max() <= 1e-13


def test_oracle_deposit_exact_large_node_sums():
    """Node totals far beyond 2^63 units of 2^-52 (a node column summing to more than 2048):
    the checker stays exact where one int64 accumulator would wrap."""
    from fractions import Fraction

    rng = np.random.default_rng(9)
    n_cells, n_nodes, n = 3, 6, 12000
    c2n = np.array([[0, 1, 2, 3], [0, 1, 4, 5], [0, 2, 3, 5]], np.int32)
    p2c = rng.integers(0, n_cells, n).astype(np.int32)
    lc = rng.uniform(0.5, 1.0, (n, 4))
    lc[:50, 2] = -rng.uniform(0, 0.3, 50)
    got = O.deposit_exact(lc, p2c, c2n, n_nodes)
    units = np.floor(lc * 2.0 ** 52).astype(np.int64)
    ref = [0] * n_nodes
    for i in range(n):
        for k in range(4):
            ref[c2n[p2c[i], k]] += int(units[i, k])
    assert max(abs(r) for r in ref) > 2 ** 63  # node 0 gathers ~9,000 weights of ~0.75
    np.testing.assert_array_equal(got, np.array([float(Fraction(r, 2 ** 52)) for r in ref]))
