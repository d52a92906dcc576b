"""Direct-hop seed on the GPU (include/oppb_dh.h) against the C oracle and the reference's
golden fixture: the structured map entry for entry, and global-move steps with the same
cells, weights, positions and counts as the oracle (node charges within 1e-12)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest
import torch

from oppb import _lib as L
from oppb.fempic import DeviceMesh, DirectHopGrid, FemPIC, HostMesh, injection_randoms, randoms_to_device
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
GOLDEN = Path(__file__).resolve().parent / "golden"


def _charge_close(gpu, ref, rtol=1e-12):
    err = np.abs(gpu - ref) / np.maximum(np.abs(ref), 1.0)
    assert err.max() <= rtol, f"node charge max rel err {err.max():.3e}"


def test_dh_map_matches_reference_golden():
    z = np.load(GOLDEN / "fempic_4x4x8_dh.npz")
    hm = HostMesh(*[float(v) if i >= 3 else int(v) for i, v in enumerate(z["dims"])])
    sp = float(z["spacing"])
    g = DirectHopGrid(hm, DeviceMesh(hm, DEV, mixed=False), sp)
    np.testing.assert_array_equal(np.array(g.dims), z["dh_dims"])
    np.testing.assert_array_equal(g.box.view(np.uint64), z["dh_box"].view(np.uint64))
    np.testing.assert_array_equal(g.map.cpu().numpy(), z["dh_map"])


@pytest.mark.parametrize("dims,spacing,expansion", [
    ((6, 5, 9, 1.0, 0.8, 1.5), 0.055, (0.2, 0.15, 0.1)),   # spacing not dividing the box, uneven widening
    ((3, 3, 5, 1.0, 1.0, 2.0), 0.5, None),                 # boxes much larger than cells
    ((4, 4, 4, 1.0, 1.0, 1.0), 0.031, None),               # boxes much smaller than cells
])
def test_dh_map_matches_oracle(dims, spacing, expansion):
    hm = HostMesh(*dims, solve_field=False)
    g = DirectHopGrid(hm, DeviceMesh(hm, DEV, mixed=False), spacing, expansion)
    exp = (4 * spacing,) * 3 if expansion is None else expansion
    dh = O.DirectHop(hm.n_pos, spacing, exp, mesh=hm)
    np.testing.assert_array_equal(np.array(g.dims), dh.dims)
    np.testing.assert_array_equal(g.box.view(np.uint64), dh.box.view(np.uint64))
    np.testing.assert_array_equal(g.map.cpu().numpy(), dh.map)


def test_dh_steps_match_reference_golden():
    """The global-move run of the reference seq backend (tests/golden/fempic_4x4x8_dh.npz):
    per-step sizes and removals, final cells, positions and weights bit for bit."""
    z = np.load(GOLDEN / "fempic_4x4x8_dh.npz")
    hm = HostMesh(*[float(v) if i >= 3 else int(v) for i, v in enumerate(z["dims"])])
    sim = FemPIC(hm, DEV, inject_per_step=int(z["inject"]), dt=float(z["dt"]), fill=str(z["fill"]),
                 fill_period=int(z["period"]), direct_hop=float(z["spacing"]))
    np.testing.assert_array_equal(sim.dist_host, z["dist"])
    for s in range(int(z["steps"])):
        r = sim.step(randoms_to_device(z["tables"][s], DEV))
        rec = z["records"][s]
        assert (r["size"], r["removed"]) == (int(rec["size"]), int(rec["removed"])), s
    got = sim.parts.host_aos()
    np.testing.assert_array_equal(got["p2c"], z["p2c"])
    np.testing.assert_array_equal(got["pos"].view(np.uint64), z["pos"].view(np.uint64))
    np.testing.assert_array_equal(got["lc"].view(np.uint64), z["lc"].view(np.uint64))
    _charge_close(sim.node_charge.cpu().numpy(), z["node_charge"])


@pytest.mark.parametrize("precision,fused_push", [("f64", True), ("f64", False), ("mixed", True), ("mixed", False)])
def test_dh_steps_match_oracle(precision, fused_push):
    """Fast particles (dt 0.2: several cells per step) on the 10x10x40-hex mesh, global move
    on, against the oracle running the same push, seed and walk."""
    hm = HostMesh(10, 10, 40, 1.0, 1.0, 4.0)
    sp = 0.1
    sim = FemPIC(hm, DEV, inject_per_step=2000, dt=0.2, precision=precision, fill="Sort_Periodic", fill_period=4,
                 fused_push=fused_push, direct_hop=sp)
    dh = O.DirectHop(hm.n_pos, sp, (4 * sp,) * 3)
    dh.map = sim.dh.map.cpu().numpy()  # (the map itself is checked above)
    orc = O.OracleFemPIC(hm, sim.dist_host, dt=0.2, fill="Sort_Periodic", fill_period=4,
                         mixed=(precision == "mixed"), dh=dh)
    removed = 0
    for s in range(24):
        rnd = injection_randoms(21, s, 2000, 0.1)
        g = sim.step(randoms_to_device(rnd, DEV))
        o = orc.step(rnd)
        assert (g["removed"], g["size"], g["visits"]) == (o["removed"], o["size"], o["visits"]), s
        removed += g["removed"]
    got = sim.parts.host_aos()
    n = orc.size
    np.testing.assert_array_equal(got["p2c"], orc.p2c[:n])
    np.testing.assert_array_equal(got["pos"].view(np.uint64), orc.pos[:n].view(np.uint64))
    if precision == "f64":
        np.testing.assert_array_equal(got["lc"].view(np.uint64), orc.lc[:n].view(np.uint64))
        _charge_close(sim.node_charge.cpu().numpy(), orc.node_charge)
    else:
        assert np.abs(got["lc"] - orc.lc[:n]).max() < 1e-5
    assert removed > 0 and n > 10_000


def test_dh_fewer_visits_for_fast_particles():
    """What the seed is for: with particles crossing several cells per step the walks are
    shorter from the grid's cell than from the previous cell (same end cells)."""
    hm = HostMesh(10, 10, 40, 1.0, 1.0, 4.0)
    a = FemPIC(hm, DEV, inject_per_step=2000, dt=0.4, direct_hop=0.1)
    b = FemPIC(hm, DEV, inject_per_step=2000, dt=0.4)
    va = vb = 0
    for s in range(8):
        rnd = randoms_to_device(injection_randoms(4, s, 2000, 0.1), DEV)
        ra, rb = a.step(rnd), b.step(rnd)
        assert (ra["size"], ra["removed"]) == (rb["size"], rb["removed"]), s
        va, vb = va + ra["visits"], vb + rb["visits"]
    np.testing.assert_array_equal(a.parts.host_aos()["p2c"], b.parts.host_aos()["p2c"])
    assert va < vb


def test_dh_full_size_spot_check():
    """The 48x48x192-hex mesh (2,654,208 cells) with spacing 1/48: the GPU map against the
    oracle's search over all cells on sampled boxes (inside, on and outside the mesh)."""
    hm = HostMesh(48, 48, 192, 1.0, 1.0, 4.0, solve_field=False)
    sp = 1.0 / 48
    g = DirectHopGrid(hm, DeviceMesh(hm, DEV, mixed=False), sp)
    gmap = g.map.cpu().numpy()
    dh = O.DirectHop(hm.n_pos, sp, (4 * sp,) * 3)
    np.testing.assert_array_equal(np.array(g.dims), dh.dims)
    inside = np.flatnonzero(gmap != O.REMOVED)
    outside = np.flatnonzero(gmap == O.REMOVED)
    assert len(inside) >= hm.n_cells // 6 and len(outside) > 0
    rng = np.random.default_rng(0)
    assert gmap[inside].max() < hm.n_cells
    idx = np.concatenate([rng.choice(inside, 24, replace=False), rng.choice(outside, 4, replace=False),
                          inside[:2], inside[-2:]])
    np.testing.assert_array_equal(gmap[idx], dh.boxes(hm, idx))


def test_dh_move_ex_errors():
    hm = HostMesh(3, 3, 5, 1.0, 1.0, 2.0, solve_field=False)
    sim = FemPIC(hm, DEV, inject_per_step=100, direct_hop=0.25)
    lib = L.load()
    v = sim.parts.view()
    st = sim.parts.status.data_ptr()
    bad = [L.MoveOptions(precision=7, deposit=1), L.MoveOptions(precision=0, deposit=0, push=1),
           L.MoveOptions(precision=1, deposit=0)]
    for o in bad:
        assert lib.oppb_move_ex(C.byref(sim.mesh.s), C.byref(v), C.byref(o), sim.node_charge.data_ptr(), st, 64,
                                None, 0, None) == L.OPPB_ERR_ARG
    g = L.DhGrid.from_buffer_copy(bytes(sim.dh.g))
    g.map = None
    o = L.MoveOptions(precision=0, deposit=1, dh=C.pointer(g))
    assert lib.oppb_move_ex(C.byref(sim.mesh.s), C.byref(v), C.byref(o), sim.node_charge.data_ptr(), st, 64,
                            None, 0, None) == L.OPPB_ERR_ARG
    assert lib.oppb_dh_grid_init(None, 0, 0.1, None, C.byref(g)) == L.OPPB_ERR_ARG
