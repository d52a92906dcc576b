"""Parity of the CabanaPIC move + current deposit kernel (through the C ABI) with the oracle
and with the reference's own outputs (golden fixture): positions, momenta, streaks, cells
and call counts bit-exact; the 12 accumulators, summed with FP64 atomics in a different
order, within CUR_RTOL of the largest accumulator magnitude.  Each test runs on the kernel
compiled with the compiler's register count and for 4 and 5 resident CTAs per SM."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oppb import _lib as L
from oppb.cabana import CabanaDevice, Deck, HexMesh, synthetic_interp, two_stream
from oracle import cabana as OC

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
CUR_RTOL = 1e-12
GOLDEN = Path(__file__).resolve().parent / "golden" / "cabana_4x5x6.npz"


@pytest.fixture(autouse=True, params=[0, 4, 5], ids=["occ-default", "occ4", "occ5"])
def occupancy(request):
    """Every test runs on every compilation of the kernel (oppb_tuning.cabana_occupancy)."""
    L.set_tuning(cabana_occupancy=request.param)
    yield request.param
    L.set_tuning(cabana_occupancy=4)


class _K:
    """Constants object for CabanaDevice.move_deposit from explicit values."""

    def __init__(self, qdt_2mc, cdt_d, qsp):
        self.qdt_2mc, self.cdt_d, self.qsp = qdt_2mc, tuple(cdt_d), qsp

    def consts(self):
        import ctypes as C
        return L.CabanaConsts(self.qdt_2mc, (C.c_double * 3)(*self.cdt_d), self.qsp)


def _bits_equal(a, b, name):
    np.testing.assert_array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8), err_msg=name)


def _acc_close(got, ref):
    scale = max(np.abs(ref).max(), 1e-300)
    err = np.abs(got - ref).max() / scale
    assert err <= CUR_RTOL, f"accumulator max err {err:.2e} of max |acc|"


def _run_gpu(mesh, interp, pos, vel, streak, w, p2c, k, calls=1, max_hops=4096, precision="f64"):
    dev = CabanaDevice(mesh, DEV, len(p2c), precision=precision)
    dev.set_interp(interp)
    dev.set_particles(pos, vel, streak, w, p2c)
    for _ in range(calls):
        dev.move_deposit(k, max_hops=max_hops)
    torch.cuda.synchronize()
    return dev.host(), dev.status_host()


def _run_oracle(mesh, interp, pos, vel, streak, w, p2c, k, calls=1, precision="f64"):
    a = {"pos": pos.copy(), "vel": vel.astype(np.float32 if precision == "mixed" else np.float64),
         "streak": streak.copy(), "p2c": p2c.copy()}
    fn = OC.move_deposit_mixed if precision == "mixed" else OC.move_deposit
    visits = 0
    for _ in range(calls):
        acc = np.zeros((mesh.n_cells, 12))
        visits = fn(a["pos"], a["vel"], a["streak"], w, a["p2c"], mesh.c2ngc, interp, acc, k.qdt_2mc,
                    np.array(k.cdt_d), k.qsp)
    a["acc"] = acc
    return a, visits


def test_matches_reference_golden():
    z = np.load(GOLDEN)
    mesh = HexMesh(*[int(v) for v in z["dims"]])
    k = _K(float(z["qdt_2mc"]), z["cdt_d"], float(z["qsp"]))
    got, st = _run_gpu(mesh, z["interp"], z["pos"], z["vel"], z["streak"], z["weight"], z["p2c"], k,
                       calls=int(z["calls"]))
    assert st.error == 0
    for name in ("pos", "vel", "streak", "p2c"):
        _bits_equal(got[name], z["ref_" + name], name)
    _acc_close(got["acc"], z["ref_acc"])


@pytest.mark.parametrize("n,seed,scale", [(1, 0, 2.0), (33, 1, 2.0), (5000, 2, 0.5), (200_003, 3, 2.5)])
def test_matches_oracle_random(n, seed, scale):
    mesh = HexMesh(6, 5, 7)
    rng = np.random.default_rng(seed)
    interp = synthetic_interp(mesh, seed + 100, e_scale=0.3, b_scale=0.4)
    p2c = np.sort(rng.choice(mesh.interior, n)).astype(np.int32)
    pos = rng.uniform(-1, 1, (n, 3))
    vel = rng.normal(0, scale, (n, 3))
    if n > 200:
        pos[:60, 1] = 1.0  # on a face
        vel[60:120, 0] = 0.0  # zero component: the 3.4e38 branch
    w = rng.uniform(0.1, 2.0, n)
    k = _K(-0.27, (1.4, 0.8, 2.2), -1.0)
    streak = np.zeros((n, 3))
    got, st = _run_gpu(mesh, interp, pos, vel, streak, w, p2c, k)
    ref, visits = _run_oracle(mesh, interp, pos, vel, streak, w, p2c, k)
    assert st.error == 0 and int(st.total_visits) == visits
    for name in ("pos", "vel", "streak", "p2c"):
        _bits_equal(got[name], ref[name], name)
    _acc_close(got["acc"], ref["acc"])


def test_two_stream_steps_match_oracle():
    """The workload's own construction at small size, five successive calls."""
    mesh = HexMesh(4, 4, 16)
    deck = Deck(4, 4, 16, 1.0, 1.0, 4.0, nppc=64, courant_frac=0.5)
    pos, vel, streak, w, p2c = two_stream(mesh, deck, 0.2, 0.01, seed=5)
    interp = synthetic_interp(mesh, 6)
    got, st = _run_gpu(mesh, interp, pos, vel, streak, w, p2c, deck, calls=5)
    ref, visits = _run_oracle(mesh, interp, pos, vel, streak, w, p2c, deck, calls=5)
    assert st.error == 0 and int(st.total_visits) == visits
    for name in ("pos", "vel", "streak", "p2c"):
        _bits_equal(got[name], ref[name], name)
    _acc_close(got["acc"], ref["acc"])


def test_errors_reported():
    mesh = HexMesh(3, 3, 3)
    interp = synthetic_interp(mesh, 1)
    n = 64
    rng = np.random.default_rng(3)
    p2c = np.full(n, mesh.interior[0], np.int32)
    p2c[17] = mesh.n_cells + 3
    pos, vel = rng.uniform(-1, 1, (n, 3)), rng.normal(0, 0.1, (n, 3))
    k = _K(-0.2, (0.5, 0.5, 0.5), -1.0)
    _, st = _run_gpu(mesh, interp, pos, vel, np.zeros((n, 3)), np.ones(n), p2c, k)
    assert st.error == L.OPPB_ERR_CELL_RANGE and st.error_index == 17
    # a long streak with a hop bound of 2 calls
    vel2 = np.zeros((1, 3))
    vel2[0, 2] = 50.0
    _, st = _run_gpu(mesh, interp, np.zeros((1, 3)), vel2, np.zeros((1, 3)), np.ones(1),
                     np.array([mesh.interior[0]], np.int32), _K(-0.2, (3.0, 3.0, 3.0), -1.0), max_hops=2)
    assert st.error == L.OPPB_ERR_HOP_LIMIT and st.error_index == 0


# ---------------------------------------------------------------- FP32-momentum form

@pytest.mark.parametrize("n,seed,scale", [(1, 0, 2.0), (5000, 2, 0.5), (200_003, 3, 2.5)])
def test_mixed_matches_oracle_random(n, seed, scale):
    """FP32 momentum: bit-exact against the oracle running the same FP32 push (positions,
    FP32 momenta, streaks, cells, call counts); accumulators within CUR_RTOL."""
    mesh = HexMesh(6, 5, 7)
    rng = np.random.default_rng(seed)
    interp = synthetic_interp(mesh, seed + 100, e_scale=0.3, b_scale=0.4)
    p2c = np.sort(rng.choice(mesh.interior, n)).astype(np.int32)
    pos = rng.uniform(-1, 1, (n, 3))
    vel = rng.normal(0, scale, (n, 3)).astype(np.float32)
    if n > 200:
        pos[:60, 1] = 1.0
        vel[60:120, 0] = 0.0
    w = rng.uniform(0.1, 2.0, n)
    k = _K(-0.27, (1.4, 0.8, 2.2), -1.0)
    streak = np.zeros((n, 3))
    got, st = _run_gpu(mesh, interp, pos, vel, streak, w, p2c, k, precision="mixed")
    ref, visits = _run_oracle(mesh, interp, pos, vel, streak, w, p2c, k, precision="mixed")
    assert st.error == 0 and int(st.total_visits) == visits
    assert got["vel"].dtype == np.float32
    for name in ("pos", "vel", "streak", "p2c"):
        _bits_equal(got[name], ref[name], name)
    _acc_close(got["acc"], ref["acc"])


def test_mixed_two_stream_steps_match_oracle_and_track_fp64():
    """The workload's construction, five calls: the FP32-momentum form equals its oracle bit for
    bit and stays close to the FP64 reference form started from the same (FP32-rounded)
    momenta: momenta within 1e-5 of the largest, currents within 1e-4 of the largest, and all
    but a few cells the same."""
    mesh = HexMesh(4, 4, 16)
    deck = Deck(4, 4, 16, 1.0, 1.0, 4.0, nppc=64, courant_frac=0.5)
    pos, vel, streak, w, p2c = two_stream(mesh, deck, 0.2, 0.01, seed=5)
    vel32 = vel.astype(np.float32)
    interp = synthetic_interp(mesh, 6)
    got, st = _run_gpu(mesh, interp, pos, vel32, streak, w, p2c, deck, calls=5, precision="mixed")
    ref, visits = _run_oracle(mesh, interp, pos, vel32, streak, w, p2c, deck, calls=5, precision="mixed")
    assert st.error == 0 and int(st.total_visits) == visits
    for name in ("pos", "vel", "streak", "p2c"):
        _bits_equal(got[name], ref[name], name)
    _acc_close(got["acc"], ref["acc"])
    f64, _ = _run_oracle(mesh, interp, pos, vel32.astype(np.float64), streak, w, p2c, deck, calls=5)
    assert np.abs(got["vel"] - f64["vel"]).max() <= 1e-5 * np.abs(f64["vel"]).max()
    assert np.abs(got["acc"] - f64["acc"]).max() <= 1e-4 * np.abs(f64["acc"]).max()
    assert (got["p2c"] != f64["p2c"]).mean() <= 1e-3


def _cols(*arrays):
    """ctypes arrays of device column pointers."""
    import ctypes as C
    return (C.c_void_p * len(arrays))(*[a.data_ptr() for a in arrays])


def test_cell_loops_equal_their_expressions_bit_for_bit():
    """The CabanaPIC cell loops of include/oppb_cabana.h (interpolate, accumulate, the two leapfrog
    updates, the ghost copies and folds) against the user kernels' expressions evaluated in numpy
    in the same order (each operation rounded on its own, as in apps/app_cabanapic/kernels.h):
    equal bit for bit on random fields, random neighbour columns and random masks, cells outside
    the masks untouched; the energy within 1e-13 of numpy's sum (its order differs)."""
    import ctypes as C
    lib = L.load()
    rng = np.random.default_rng(11)
    n, s = 5000, 5007
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    E, B = rng.normal(size=(3, s)), rng.normal(size=(3, s))
    acc = rng.normal(size=(12, s))
    nb = [rng.integers(0, n, n).astype(np.int32) for _ in range(9)]
    ghost = (rng.random(s) < 0.2).astype(np.int32)
    right = (rng.random(s) < 0.7).astype(np.int32)
    dE, dB, dacc = t(E), t(B), t(acc)
    dnb = [t(c) for c in nb]
    dghost, dright = t(ghost), t(right)
    m = ghost[:n] == 0
    c = np.arange(n)

    # interpolate_mesh_fields_kernel
    interp = np.full((18, s), 7.0)
    dinterp = t(interp)
    L.check("interp", lib.oppb_cabana_interpolate(n, s, dE.data_ptr(), dB.data_ptr(), _cols(*dnb[:6]),
                                                  _cols(*dnb[6:]), dinterp.data_ptr(), dghost.data_ptr(), None))
    q, h = 1.0 / 4.0, 1.0 / 2.0
    cx, cy, cz, cxy, cyz, cxz = nb[:6]
    want = interp.copy()
    for k0, (w0, w1, w2, w3) in ((0, (E[0, c], E[0, cy], E[0, cz], E[0, cyz])),
                                 (4, (E[1, c], E[1, cz], E[1, cx], E[1, cxz])),
                                 (8, (E[2, c], E[2, cx], E[2, cy], E[2, cxy]))):
        vals = (q * ((w3 + w0) + (w1 + w2)), q * ((w3 - w0) + (w1 - w2)), q * ((w3 - w0) - (w1 - w2)),
                q * ((w3 + w0) - (w1 + w2)))
        for k, v in enumerate(vals):
            want[k0 + k, :n] = np.where(m, v, want[k0 + k, :n])
    for d, up in enumerate(nb[6:]):
        w0, w1 = B[d, c], B[d, up]
        want[12 + 2 * d, :n] = np.where(m, h * (w1 + w0), want[12 + 2 * d, :n])
        want[13 + 2 * d, :n] = np.where(m, h * (w1 - w0), want[13 + 2 * d, :n])
    np.testing.assert_array_equal(dinterp.cpu().numpy().view(np.uint64), want.view(np.uint64))

    # accumulate_current_to_cells_kernel
    J = np.full((3, s), 5.0)
    dJ = t(J)
    coef = (C.c_double * 3)(0.3, -1.7, 2.9)
    L.check("acc", lib.oppb_cabana_accumulate(n, s, dJ.data_ptr(), dacc.data_ptr(), _cols(*dnb[:6]),
                                              dright.data_ptr(), coef, None))
    xd, yd, zd, xyd, yzd, xzd = nb[:6]
    r = right[:n] == 1
    want = J.copy()
    want[0, :n] = np.where(r, 0.3 * (((acc[0, c] + acc[1, yd]) + acc[2, zd]) + acc[3, yzd]), J[0, :n])
    want[1, :n] = np.where(r, -1.7 * (((acc[4, c] + acc[5, zd]) + acc[6, xd]) + acc[7, xzd]), J[1, :n])
    want[2, :n] = np.where(r, 2.9 * (((acc[8, c] + acc[9, xd]) + acc[10, yd]) + acc[11, xyd]), J[2, :n])
    np.testing.assert_array_equal(dJ.cpu().numpy().view(np.uint64), want.view(np.uint64))

    # half_advance_b_kernel, then advance_e_kernel (B and J from above)
    p = (C.c_double * 3)(0.41, 0.57, 0.33)
    px, py, pz = 0.41, 0.57, 0.33
    L.check("hab", lib.oppb_cabana_half_advance_b(n, s, _cols(*dnb[:3]), dE.data_ptr(), dB.data_ptr(),
                                                  dghost.data_ptr(), p, None))
    Bw = B.copy()
    ux, uy, uz = nb[:3]
    Bw[0, :n] = np.where(m, B[0, c] - ((0.5 * py) * (E[2, uy] - E[2, c]) - (0.5 * pz) * (E[1, uz] - E[1, c])), B[0, :n])
    Bw[1, :n] = np.where(m, B[1, c] - ((0.5 * pz) * (E[0, uz] - E[0, c]) - (0.5 * px) * (E[2, ux] - E[2, c])), B[1, :n])
    Bw[2, :n] = np.where(m, B[2, c] - ((0.5 * px) * (E[1, ux] - E[1, c]) - (0.5 * py) * (E[0, uy] - E[0, c])), B[2, :n])
    np.testing.assert_array_equal(dB.cpu().numpy().view(np.uint64), Bw.view(np.uint64))
    Jw = want
    dt = 0.123
    L.check("ae", lib.oppb_cabana_advance_e(n, s, _cols(*dnb[3:6]), dB.data_ptr(), dJ.data_ptr(), dE.data_ptr(),
                                            dright.data_ptr(), p, dt, None))
    lx, ly, lz = nb[3:6]
    Ew = E.copy()
    Ew[0, :n] = np.where(r, E[0, c] + ((-dt * Jw[0, c]) + (py * (Bw[2, c] - Bw[2, ly]) - pz * (Bw[1, c] - Bw[1, lz]))),
                         E[0, :n])
    Ew[1, :n] = np.where(r, E[1, c] + ((-dt * Jw[1, c]) + (pz * (Bw[0, c] - Bw[0, lz]) - px * (Bw[2, c] - Bw[2, lx]))),
                         E[1, :n])
    Ew[2, :n] = np.where(r, E[2, c] + ((-dt * Jw[2, c]) + (px * (Bw[1, c] - Bw[1, lx]) - py * (Bw[0, c] - Bw[0, ly]))),
                         E[2, :n])
    np.testing.assert_array_equal(dE.cpu().numpy().view(np.uint64), Ew.view(np.uint64))

    # update_ghosts_B_kernel / update_ghosts_kernel: sources in the first half, distinct targets in
    # the second, the same dat read and written as the app does
    half_n = n // 2
    to_map = np.arange(n, dtype=np.int32)
    to_map[:half_n] = half_n + rng.permutation(n - half_n)[:half_n]
    mask = np.zeros((6, s), dtype=np.int32)
    mask[:, :half_n] = (rng.random((6, half_n)) < 0.5)
    dmask, dmap = t(mask), t(to_map)
    F = rng.normal(size=(3, s))
    for m_idx, dim in ((2, -1), (4, 1)):
        dF = t(F)
        L.check("ghosts", lib.oppb_cabana_update_ghosts(n, s, dmask.data_ptr(), m_idx, dF.data_ptr(), dF.data_ptr(),
                                                        dmap.data_ptr(), dim, None))
        Fw = F.copy()
        src = np.nonzero(mask[m_idx, :n] == 1)[0]
        for d in (range(3) if dim < 0 else [dim]):
            Fw[d, to_map[src]] = F[d, src] if dim < 0 else F[d, to_map[src]] + F[d, src]
        np.testing.assert_array_equal(dF.cpu().numpy().view(np.uint64), Fw.view(np.uint64))

    # compute_energy_kernel
    ws = torch.empty(lib.oppb_cabana_energy_workspace_bytes(), dtype=torch.uint8, device=DEV)
    out = torch.tensor([0.5], dtype=torch.float64, device=DEV)
    L.check("energy", lib.oppb_cabana_energy(n, s, dghost.data_ptr(), dE.data_ptr(), out.data_ptr(),
                                             ws.data_ptr(), ws.numel(), None))
    fx, fy, fz = Ew[0, :n], Ew[1, :n], Ew[2, :n]
    ref = 0.5 + float(np.sum(np.where(m, (fx * fx + fy * fy) + fz * fz, 0.0)))
    assert abs(float(out.item()) - ref) <= 1e-13 * ref
