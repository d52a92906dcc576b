"""NESO-advection kernels through the C ABI: a batch of independent instances of different
meshes, particle counts and constants, advanced by one persistent launch per step, against the
oracle run on every instance alone; positions, move directions, cells and move-call counts
bit-exact.  Also the reference's own outputs (golden fixture), the separate update_pos / move
loops, CUDA-graph replay, and the error paths."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oppb import _lib as L
from oppb.advec import AdvecBatchDevice, AdvecMesh, particles
from oracle import advec as OA

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
GOLDEN = Path(__file__).resolve().parent / "golden" / "advec_13x9.npz"

# (nx, ny, cell_width, dt, ppc, v_sd): extents >= 1 on both axes (the reference's wrap needs it)
INSTANCES = [(13, 9, 0.7, 0.35, 30, 2.0), (40, 17, 1.0, 0.5, 7, 0.6), (7, 33, 0.3, 0.2, 11, 1.5),
             (64, 64, 1.0, 0.5, 50, 0.5), (4, 4, 1.0, 0.8, 3, 4.0)]


def _build(specs, seed0=0):
    meshes = [AdvecMesh(nx, ny, cw) for nx, ny, cw, _, _, _ in specs]
    host = [particles(m, ppc, v_sd, seed0 + k) for k, (m, (_, _, _, _, ppc, v_sd)) in enumerate(zip(meshes, specs))]
    dev = AdvecBatchDevice(meshes, [len(h[3]) for h in host], [s[3] for s in specs], DEV)
    for k, h in enumerate(host):
        dev.set_instance(k, *h)
    return meshes, host, dev


def _oracle(meshes, host, specs, steps):
    out, visits = [], 0
    for m, (pos, vel, mdir, p2c), s in zip(meshes, host, specs):
        pos, mdir, p2c = pos.copy(), mdir.copy(), p2c.copy()
        for _ in range(steps):
            visits += OA.steps(pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, s[3], m.extents, m.cell_width, 1)
        out.append({"pos": pos, "mdir": mdir, "p2c": p2c})
    return out, visits


def _assert_same(dev, ref):
    for k, r in enumerate(ref):
        got = dev.host_instance(k)
        np.testing.assert_array_equal(got["pos"].view(np.uint64), r["pos"].view(np.uint64), err_msg=f"pos {k}")
        np.testing.assert_array_equal(got["mdir"], r["mdir"], err_msg=f"mdir {k}")
        np.testing.assert_array_equal(got["p2c"], r["p2c"], err_msg=f"p2c {k}")


def test_batch_step_matches_oracle_per_instance():
    steps = 6
    meshes, host, dev = _build(INSTANCES)
    dev.zero_status()
    for _ in range(steps):
        dev.step()
    torch.cuda.synchronize()
    st = dev.status_host()
    ref, visits = _oracle(meshes, host, INSTANCES, steps)
    assert st.error == 0 and int(st.total_visits) == visits
    _assert_same(dev, ref)


def test_matches_reference_golden():
    z = np.load(GOLDEN)
    m = AdvecMesh(int(z["nx"]), int(z["ny"]), float(z["cell_width"]))
    dev = AdvecBatchDevice([m], [len(z["p2c"])], [float(z["dt"])], DEV)
    dev.set_instance(0, z["pos"], z["vel"], z["mdir"], z["p2c"])
    for _ in range(int(z["steps"])):
        dev.step()
    torch.cuda.synchronize()
    got = dev.host_instance(0)
    np.testing.assert_array_equal(got["pos"].view(np.uint64), z["ref_pos"].view(np.uint64))
    np.testing.assert_array_equal(got["mdir"], z["ref_mdir"])
    np.testing.assert_array_equal(got["p2c"], z["ref_p2c"])


def test_separate_loops_equal_fused_step():
    meshes, host, dev_a = _build(INSTANCES, seed0=20)
    _, _, dev_b = _build(INSTANCES, seed0=20)
    for _ in range(4):
        dev_a.step()
        dev_b.update_pos()
        dev_b.move()
    torch.cuda.synchronize()
    for k in range(len(INSTANCES)):
        a, b = dev_a.host_instance(k), dev_b.host_instance(k)
        for name in ("pos", "mdir", "p2c"):
            np.testing.assert_array_equal(a[name], b[name], err_msg=f"{name} {k}")
    assert int(dev_a.status_host().total_visits) == int(dev_b.status_host().total_visits)


def test_cuda_graph_replay_equals_launches():
    meshes, host, dev_a = _build(INSTANCES, seed0=40)
    _, _, dev_b = _build(INSTANCES, seed0=40)
    dev_a.zero_status()
    dev_b.zero_status()
    dev_a.step()  # sizes the persistent grid outside the capture
    dev_b.step()
    g = dev_b.capture(3)
    for _ in range(6):
        dev_a.step()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for k in range(len(INSTANCES)):
        a, b = dev_a.host_instance(k), dev_b.host_instance(k)
        for name in ("pos", "mdir", "p2c"):
            np.testing.assert_array_equal(a[name], b[name], err_msg=f"{name} {k}")
    assert int(dev_a.status_host().total_visits) == int(dev_b.status_host().total_visits)


def test_errors_reported():
    m = AdvecMesh(6, 6, 1.0)
    pos, vel, mdir, p2c = particles(m, 4, 0.5, 1)
    p2c[9] = 1000
    dev = AdvecBatchDevice([m], [len(p2c)], [0.5], DEV)
    dev.set_instance(0, pos, vel, mdir, p2c)
    dev.zero_status()
    dev.step()
    st = dev.status_host()
    assert st.error == L.OPPB_ERR_CELL_RANGE and st.error_index == 9
    # extents below 1 break the reference's wrap: the walk around the ring ends at the hop bound
    m2 = AdvecMesh(2, 2, 0.25)
    pos, vel, mdir, p2c = particles(m2, 2, 0.0, 2)
    vel[0] = (-40.0, 0.0)
    dev2 = AdvecBatchDevice([m2], [len(p2c)], [0.1], DEV)
    dev2.set_instance(0, pos, vel, mdir, p2c)
    dev2.zero_status()
    dev2.step(max_hops=64)
    st = dev2.status_host()
    assert st.error == L.OPPB_ERR_HOP_LIMIT and st.error_index == 0


def test_verify_kernel_invariant_on_a_large_batch():
    """The reference's verify_kernel (apps/app_neso_advection/kernels.h:115-151) after many steps
    of a batch of larger instances: every particle's position lies in the closed box
    [ix w, ix w + w] x [iy w, iy w + w] of its cell (ix, iy) = (cell mod nx, cell div nx), so the
    incorrect count is 0."""
    specs = [(128, 96, 1.0, 0.5, 60, 0.5), (200, 64, 0.25, 0.1, 25, 1.0), (33, 257, 0.7, 0.3, 40, 0.8),
             (256, 256, 1.0, 0.5, 20, 0.5)]
    meshes, _, dev = _build(specs, seed0=40)
    dev.zero_status()
    for _ in range(40):
        dev.step()
    torch.cuda.synchronize()
    assert dev.status_host().error == 0
    for k, m in enumerate(meshes):
        got = dev.host_instance(k)
        ix, iy = got["p2c"] % m.nx, got["p2c"] // m.nx
        w = m.cell_width
        llx, lly = ix * w, iy * w  # the reference's boundary_ll, in FP64
        x, y = got["pos"][:, 0], got["pos"][:, 1]
        incorrect = (ix < 0) | (iy < 0) | (x < llx) | (x > llx + w) | (y < lly) | (y > lly + w)
        assert int(incorrect.sum()) == 0, (k, int(incorrect.sum()))


def test_ensemble_of_64_over_500_steps_under_graph_matches_oracle():
    """Config 5 at its own scale and length: 64 instances with sides drawn from U{64..512} (the
    benchmark's seeded draw), |v dt| <= 0.5 cell, 500 steps advanced as 50 replays of a 10-step
    CUDA graph of the persistent launch; positions, move directions and cells of every
    instance bit-exact against the oracle run on each instance alone (worker processes).
    Particles per cell are drawn from U{1..3} instead of U{10..200}, so that the oracle's
    ~6e9 particle-steps finish in about a minute; the kernels, the in-order work counter and
    the graph see the same 64 uneven meshes."""
    import multiprocessing as mp
    import os

    rng = np.random.default_rng(5)
    sides = rng.integers(64, 513, 64)
    ppcs = rng.integers(1, 4, 64)
    specs = [(int(sd), int(sd), 1.0, 0.5, int(pc), 0.5) for sd, pc in zip(sides, ppcs)]
    meshes = [AdvecMesh(nx, ny, cw) for nx, ny, cw, _, _, _ in specs]
    host = [particles(m, s[4], s[5], 5000 + k, v_clip=1.0) for k, (m, s) in enumerate(zip(meshes, specs))]
    steps = 500
    jobs = [(h[0], h[1], h[2], h[3], m.c2c, m.c_pos_ll, s[3], np.array(m.extents, np.float64), m.cell_width, steps)
            for m, h, s in zip(meshes, host, specs)]
    ctx = mp.get_context("spawn")  # workers import only the oracle
    pool = ctx.Pool(max(1, min(len(jobs), len(os.sched_getaffinity(0)) - 1)))
    pending = pool.map_async(OA.steps_job, jobs, chunksize=1)
    dev = AdvecBatchDevice(meshes, [len(h[3]) for h in host], [s[3] for s in specs], DEV)
    for k, h in enumerate(host):
        dev.set_instance(k, *h)
    dev.zero_status()
    dev.step()  # sizes the persistent grid outside the capture
    g = dev.capture(10)
    for _ in range((steps - 1) // 10):
        g.replay()
    for _ in range((steps - 1) % 10):
        dev.step()
    torch.cuda.synchronize()
    assert dev.status_host().error == 0
    ref = pending.get(timeout=1800)
    pool.close()
    pool.join()
    assert sum(len(h[3]) for h in host) > 5_000_000
    _assert_same(dev, [{"pos": r[0], "mdir": r[1], "p2c": r[2]} for r in ref])
