"""The C-ABI library without a GPU: it loads, exports every function the headers in
include/ declare, and validates arguments before touching the device."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from oppb import _lib as L

INCLUDE = Path(__file__).resolve().parent.parent / "include"


def declared_functions():
    names = set()
    for h in sorted(INCLUDE.glob("oppb*.h")):  # every header of the C ABI library
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(oppb_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_status_strings():
    lib = L.load()
    assert b"sm_100a" in lib.oppb_version()
    for s in range(8):
        assert lib.oppb_status_string(s)
    assert lib.oppb_status_string(99) == b"unknown status"


def test_argument_validation_without_device():
    lib = L.load()
    assert lib.oppb_move_f64(None, None, None, 16, None) == L.OPPB_ERR_ARG
    m = L.TetMesh(10, 10, None, None, None, None, None, None)
    p = L.Particles(5, 4, None, None, None, None, None)  # stride < size
    assert lib.oppb_move_f64(C.byref(m), C.byref(p), None, 16, None) == L.OPPB_ERR_ARG
    assert lib.oppb_push_f64(C.byref(m), C.byref(p), 1.0, 0.01, None) == L.OPPB_ERR_ARG
    assert lib.oppb_hole_fill(-1, 0, None, 0, 0, None, None, 0, None) == L.OPPB_ERR_ARG
    assert lib.oppb_hole_fill(10, 0, None, 10, 0, None, None, 0, None) == L.OPPB_OK  # nothing removed
    assert lib.oppb_sort_by_cell(10, 0, 10, 1, None, 0, None, None, 0, None) == L.OPPB_ERR_ARG


def test_workspace_queries():
    lib = L.load()
    assert lib.oppb_hole_fill_workspace_bytes(0, 0) > 0
    small = lib.oppb_sort_workspace_bytes(1000, 100)
    big = lib.oppb_sort_workspace_bytes(50_000_000, 2_654_208)
    assert big > 5 * 4 * 50_000_000 > small
    assert lib.oppb_sort_workspace_bytes(-1, 5) == 0


def test_kernel_launch_counter_starts_at_zero_without_launches():
    assert L.load().oppb_kernel_launches() >= 0


@pytest.mark.parametrize("n", [1, 1000])
def test_mesh_bytes(n):
    out = (C.c_size_t * 6)()
    L.load().oppb_tet_mesh_bytes(n, out)
    assert list(out) == [128 * n, 32 * n, 16 * n, 32 * n, 64 * n, 32 * n]


def test_declared_functions_cover_every_header():
    names = declared_functions()
    for n in ("oppb_move_ex", "oppb_dh_build", "oppb_cabana_move_deposit", "oppb_advec_step"):
        assert n in names


@pytest.mark.parametrize("dims,spacing,expansion", [
    ((4, 4, 8, 1.0, 1.0, 2.0), 0.1, (0.4, 0.4, 0.4)),
    ((5, 3, 6, 1.0, 0.6, 1.2), 0.07, (0.3, 0.2, 0.25)),
    ((48, 48, 192, 1.0, 1.0, 4.0), 1.0 / 48, (4.0 / 48,) * 3),
])
def test_dh_grid_init_matches_oracle(dims, spacing, expansion):
    """The host half of the direct-hop set-up (bounding box and box counts) equals the
    oracle's restatement of the reference, bit for bit, without a GPU."""
    import numpy as np

    from oppb.fempic import HostMesh
    from oracle import oracle as O

    hm = HostMesh(*dims, solve_field=False)
    g = L.DhGrid()
    exp = np.array(expansion)
    assert L.load().oppb_dh_grid_init(np.ascontiguousarray(hm.n_pos).ctypes.data, hm.n_nodes, spacing,
                                      exp.ctypes.data, C.byref(g)) == L.OPPB_OK
    o = O.DirectHop(hm.n_pos, spacing, expansion)
    assert list(g.dims) == list(o.dims) and g.size == o.size
    box = np.array(list(g.min) + list(g.max))
    np.testing.assert_array_equal(box.view(np.uint64), o.box.view(np.uint64))
    assert g.inv_spacing == 1.0 / spacing


def test_dh_and_move_ex_argument_validation():
    lib = L.load()
    g = L.DhGrid()
    one = (C.c_double * 3)(0.0, 0.0, 0.0)
    pts = (C.c_double * 3)(0.0, 0.0, 0.0)
    assert lib.oppb_dh_grid_init(pts, 1, 0.0, one, C.byref(g)) == L.OPPB_ERR_ARG      # spacing 0
    assert lib.oppb_dh_grid_init(pts, 0, 0.1, one, C.byref(g)) == L.OPPB_ERR_ARG      # no nodes
    assert lib.oppb_dh_grid_init(pts, 1, 1e-12, (C.c_double * 3)(1.0, 1.0, 1.0), C.byref(g)) == L.OPPB_ERR_ARG
    assert lib.oppb_dh_build(None, None, C.byref(g), None, 0, None, None) == L.OPPB_ERR_ARG
    assert lib.oppb_move_ex(None, None, None, None, None, 16, None, 0, None) == L.OPPB_ERR_ARG


def test_tuning_exact_deposit_mode_and_workspace():
    """OPPB_DEPOSIT_EXACT is a valid deposit choice (unknown ones are refused) and asks for
    two 8-B integer sums per node of workspace; the other modes keep the copy sizing."""
    lib = L.load()
    before = L.Tuning()
    lib.oppb_get_tuning(C.byref(before))
    try:
        L.set_tuning(deposit=L.DEPOSIT_EXACT)
        assert lib.oppb_deposit_workspace_bytes(1000) == 16 * 1000
        assert lib.oppb_deposit_workspace_bytes(0) == 0
        L.set_tuning(deposit=L.DEPOSIT_WARP_ATOMIC, replicas=4)
        assert lib.oppb_deposit_workspace_bytes(1000) == 3 * 8 * 1000
        bad = L.Tuning()
        lib.oppb_get_tuning(C.byref(bad))
        bad.deposit = 3
        assert lib.oppb_set_tuning(C.byref(bad)) == L.OPPB_ERR_ARG
    finally:
        lib.oppb_set_tuning(C.byref(before))


def test_exact_deposit_split_bounds():
    """The fixed-point split of the exact deposit, restated in numpy: u = floor(w 2^52) (exact
    in FP64 for |w| < 2^11), a = u >> 32, b = u mod 2^32, so w = a 2^-20 + b 2^-52 + r with
    0 <= r < 2^-52, for weights of either sign, tiny negative ones (where 1 + w 2^20 is not
    exact in FP64) and the mixed path's FP32 weights widened to FP64 included."""
    rng = np.random.default_rng(3)
    tiny = -(2.0 ** -52) * (1 + rng.uniform(0, 1, 1000))
    w = np.concatenate([rng.uniform(-1e-9, 1.0 + 1e-9, 100_000), rng.uniform(-1000, 1000, 1000), tiny,
                        rng.uniform(0, 1, 1000).astype(np.float32).astype(np.float64),
                        [0.0, 1.0, -1e-10, 2 ** -52, -(2 ** -52), -(2 ** -52 + 2 ** -105)]])
    u = np.floor(w * 2.0 ** 52).astype(np.int64)
    a, b = u >> 32, u & 0xFFFFFFFF
    assert (b >= 0).all() and (b < 2 ** 32).all() and (np.abs(a) < 2 ** 31).all()
    np.testing.assert_array_equal(a * 2 ** 32 + b, u)
    # r = w - u 2^-52 in [0, 2^-52): checked in exact rational arithmetic on a sample
    from fractions import Fraction
    for x, k in zip(w[::97], u[::97]):
        r = Fraction(float(x)) - Fraction(int(k), 2 ** 52)
        assert 0 <= r < Fraction(1, 2 ** 52)
