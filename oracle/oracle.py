"""TEST INFRASTRUCTURE ONLY — Python driver of the C parity oracle (fempic_oracle.c).

Runs the FemPIC particle step in the seq backend's order and host layout (AoS numpy
arrays), following the generated main loop apps_codegen/app_fempic_cg/fempic_opp.cpp:160-215:
  opp_inc_part_count_with_distribution -> inject_ions -> reset n_charge_den -> push
  -> opp_particle_move (move_kernel, then finalize: hole fill / sort) -> deposit.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "liboppb_oracle.so"
REMOVED = 2147483647

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} missing: run op-pic_b200/build.py")
        lib = C.CDLL(str(LIB_PATH))
        vp, i32 = C.c_void_p, C.c_int32
        lib.oracle_move.restype = C.c_int64
        lib.oracle_move.argtypes = [i32, vp, vp, vp, vp, vp, vp, i32, vp, vp]
        lib.oracle_deposit.restype = None
        lib.oracle_deposit.argtypes = [i32, vp, vp, vp, vp]
        lib.oracle_push.restype = None
        lib.oracle_push.argtypes = [i32, vp, vp, vp, vp, C.c_double, C.c_double]
        lib.oracle_push_mixed.restype = None
        lib.oracle_push_mixed.argtypes = [i32, vp, vp, vp, vp, C.c_double, C.c_double]
        lib.oracle_inject.restype = None
        lib.oracle_inject.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, C.c_double, C.c_double,
                                      C.c_double, vp, vp, vp]
        lib.oracle_hole_fill.restype = i32
        lib.oracle_hole_fill.argtypes = [i32, i32, vp, i32, vp, vp, vp, vp]
        lib.oracle_sort.restype = C.c_int
        lib.oracle_sort.argtypes = [i32, i32, i32, vp, vp, i32, vp]
        lib.oracle_dh_grid_init.restype = C.c_int
        lib.oracle_dh_grid_init.argtypes = [i32, vp, C.c_double, vp, vp, vp]
        lib.oracle_dh_build.restype = None
        lib.oracle_dh_build.argtypes = [i32, vp, vp, vp, C.c_double, vp, vp]
        lib.oracle_dh_boxes.restype = None
        lib.oracle_dh_boxes.argtypes = [i32, vp, vp, vp, C.c_double, vp, i32, vp, vp]
        lib.oracle_dh_seed.restype = i32
        lib.oracle_dh_seed.argtypes = [i32, vp, vp, vp, C.c_double, vp, vp]
        _lib = lib
    return _lib


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def move(pos, lc, p2c, c2c, c_vol, c_det, n=None, max_hops=1 << 20):
    """opp_particle_move body over [0,n): returns (remove_count, total_visits, visits[n])."""
    lib = load()
    n = len(p2c) if n is None else n
    rc = C.c_int32(0)
    visits = np.zeros(max(n, 1), np.int32)
    total = lib.oracle_move(n, _p(pos), _p(lc), _p(p2c), _p(c2c), _p(c_vol), _p(c_det), max_hops,
                            C.addressof(rc), _p(visits))
    return rc.value, int(total), visits[:n]


def deposit(lc, p2c, c2n, node_charge, n=None):
    n = len(p2c) if n is None else n
    load().oracle_deposit(n, _p(lc), _p(p2c), _p(c2n), _p(node_charge))


def deposit_exact(lc, p2c, c2n, n_nodes):
    """The node charges of the deterministic deposit mode (OPPB_DEPOSIT_EXACT), from its
    definition: each weight w cut to floor(w 2^52) 2^-52 and the cut weights of a node added
    exactly (integers), the total rounded once to FP64.  lc [n][4], p2c [n] (REMOVED
    particles skipped), c2n [cells][4]; weights |w| < 2^11.  The reference sums the uncut
    weights sequentially in FP64 (deposit above); the two differ by the cut and that
    rounding."""
    keep = p2c != REMOVED
    units = np.floor(np.asarray(lc)[keep] * 2.0 ** 52).astype(np.int64)  # exact: |w| 2^52 < 2^63
    nodes = np.asarray(c2n)[p2c[keep]].ravel()
    units = units.ravel()
    # Each cut weight is hi 2^32 + lo with hi = units >> 32 (|hi| < 2^31) and lo in [0, 2^32):
    # int64 sums of either part cannot wrap for fewer than 2^31 terms, whatever a node's total.
    hi = np.zeros(n_nodes, dtype=np.int64)
    lo = np.zeros(n_nodes, dtype=np.int64)
    np.add.at(hi, nodes, units >> 32)
    np.add.at(lo, nodes, units & 0xFFFFFFFF)
    return np.array([float(int(h) * 2 ** 32 + int(l)) * 2.0 ** -52 for h, l in zip(hi, lo)])


def push(p2c, c_ef, pos, vel, qm, dt, n=None, mixed=False):
    n = len(p2c) if n is None else n
    fn = load().oracle_push_mixed if mixed else load().oracle_push
    fn(n, _p(p2c), _p(c_ef), _p(pos), _p(vel), qm, dt)


def hole_fill(size, remove_count, p2c, dats):
    """particle_hole_fill_core on AoS dats (list of 2-D arrays incl. p2c). Returns the pairs."""
    lib = load()
    ptrs = (C.c_void_p * len(dats))(*[_p(d) for d in dats])
    nbytes = np.array([d.strides[0] for d in dats], np.int32)
    pf = np.zeros(max(remove_count, 1), np.int32)
    pt = np.zeros(max(remove_count, 1), np.int32)
    n = lib.oracle_hole_fill(size, remove_count, _p(p2c), len(dats), C.addressof(ptrs), _p(nbytes), _p(pf), _p(pt))
    return pf[:n].copy(), pt[:n].copy()


def sort(size, n_cells, dats, key_dat):
    """opp_particle_sort_core with a stable order; returns the permutation."""
    lib = load()
    ptrs = (C.c_void_p * len(dats))(*[_p(d) for d in dats])
    nbytes = np.array([d.strides[0] for d in dats], np.int32)
    perm = np.zeros(max(size, 1), np.int32)
    rc = lib.oracle_sort(size, n_cells, len(dats), C.addressof(ptrs), _p(nbytes), key_dat, _p(perm))
    if rc != 0:
        raise MemoryError("oracle_sort")
    return perm[:size].copy()


class DirectHop:
    """The structured cell mapper of the global move (oracle_dh_*): grid from the node
    positions (AoS [n][3]), spacing h and expansion (3,), map built by searching all cells
    per query as the reference does (slow: small meshes only)."""

    def __init__(self, n_pos, spacing: float, expansion, mesh=None):
        lib = load()
        n_pos = np.ascontiguousarray(n_pos, np.float64)
        self.spacing = float(spacing)
        self.expansion = np.ascontiguousarray(expansion, np.float64)
        self.box = np.zeros(6)
        self.dims = np.zeros(3, np.int64)
        if lib.oracle_dh_grid_init(len(n_pos), _p(n_pos), self.spacing, _p(self.expansion), _p(self.box),
                                   _p(self.dims)) != 0:
            raise ValueError("grid too large")
        self.inv = 1.0 / self.spacing
        self.size = int(np.prod(self.dims))
        self.map = None
        if mesh is not None:
            self.build(mesh)

    def build(self, mesh) -> np.ndarray:
        self.map = np.zeros(self.size, np.int32)
        load().oracle_dh_build(mesh.n_cells, _p(np.ascontiguousarray(mesh.c_vol)),
                               _p(np.ascontiguousarray(mesh.c_det)), _p(self.box), self.spacing, _p(self.dims),
                               _p(self.map))
        return self.map

    def boxes(self, mesh, idx) -> np.ndarray:
        """Map entries of the boxes idx only (the same search, for spot checks)."""
        idx = np.ascontiguousarray(idx, np.int64)
        out = np.zeros(len(idx), np.int32)
        load().oracle_dh_boxes(mesh.n_cells, _p(np.ascontiguousarray(mesh.c_vol)),
                               _p(np.ascontiguousarray(mesh.c_det)), _p(self.box), self.spacing, _p(self.dims),
                               len(idx), _p(idx), _p(out))
        return out

    def seed(self, pos, p2c, n=None) -> int:
        """Global-move pre-pass over [0,n): p2c from the grid; returns the removals."""
        n = len(p2c) if n is None else n
        return int(load().oracle_dh_seed(n, _p(pos), _p(p2c), _p(self.box[:3].copy()), self.inv, _p(self.dims),
                                         _p(self.map)))


class OracleFemPIC:
    """The FemPIC particle step on AoS host arrays, seq-backend order.

    mesh: object with numpy arrays c2n, c2c, c_det, c_vol, c_ef, if2c, if_u, if_v, if_norm,
    if_n_pos (AoS, as the reference host layout) and n_nodes / n_cells.
    fill: 'HoleFill_All' | 'Sort_All' | 'Sort_Periodic' (opp_particle_organize_core.cpp:61-87).
    """

    def __init__(self, mesh, dist, ion_velocity=1.0, qm=1.0, dt=0.01, fill="HoleFill_All", fill_period=10,
                 alloc_mult=2.0, mixed=False, max_hops=1 << 20, dh: DirectHop | None = None, field=None):
        self.m = mesh
        self.dh = dh  # global move: every walk starts from the grid's cell
        # field phase after the deposit: (oracle.field.FieldSystem, FieldConsts, spwt, n_vol);
        # the new cell field replaces mesh.c_ef, which the next push and injection read
        self.field = field
        self.potential = None
        self.dist = np.ascontiguousarray(dist, np.int32)
        self.ion_velocity, self.qm, self.dt = ion_velocity, qm, dt
        self.fill, self.fill_period, self.alloc_mult = fill, fill_period, alloc_mult
        self.mixed = mixed
        self.max_hops = max_hops
        self.size = 0
        self.capacity = 0
        self.pos = np.zeros((0, 3))
        self.vel = np.zeros((0, 3))
        self.lc = np.zeros((0, 4))
        self.p2c = np.zeros((0,), np.int32)
        self.node_charge = np.zeros(mesh.n_nodes)
        self.iter = 0
        self.last_remove = 0
        self.last_visits = 0

    def _grow(self, count: int) -> None:
        # opp_increase_particle_count_core (opp_increase_part_count_core.cpp:35-110)
        new_size = self.size + count
        if new_size <= self.capacity:
            return
        cap = int(self.size + count * self.alloc_mult)
        for name, dim in (("pos", 3), ("vel", 3), ("lc", 4)):
            a = np.zeros((cap, dim))
            a[: self.size] = getattr(self, name)[: self.size]
            setattr(self, name, a)
        p = np.full(cap, REMOVED, np.int32)
        p[: self.size] = self.p2c[: self.size]
        self.p2c = p
        self.capacity = cap

    def inject(self, rnd_aos: np.ndarray) -> None:
        count = rnd_aos.shape[0]
        self._grow(count)
        start = self.size
        m = self.m
        load().oracle_inject(start, count, _p(self.dist), _p(m.if2c), _p(m.if_u), _p(m.if_v), _p(m.if_norm),
                             _p(m.if_n_pos), _p(m.c_ef), _p(np.ascontiguousarray(rnd_aos)), self.ion_velocity,
                             self.qm, self.dt, _p(self.pos), _p(self.vel), _p(self.p2c))
        self.size += count

    def step(self, rnd_aos: np.ndarray) -> dict:
        m = self.m
        self.inject(rnd_aos)
        self.node_charge[:] = 0.0
        push(self.p2c, m.c_ef, self.pos, self.vel, self.qm, self.dt, n=self.size, mixed=self.mixed)
        n_before = self.size
        seeded_out = self.dh.seed(self.pos, self.p2c, n=self.size) if self.dh is not None else 0
        rc, visits, _ = move(self.pos, self.lc, self.p2c, m.c2c, m.c_vol, m.c_det, n=self.size,
                             max_hops=self.max_hops)
        if visits < 0:
            raise RuntimeError("oracle: hop limit")
        rc += seeded_out
        self.finalize(rc)
        deposit(self.lc, self.p2c, m.c2n, self.node_charge, n=self.size)
        if self.field is not None:
            from oracle import field as F

            fs, consts, spwt, n_vol = self.field
            self.node_charge[:] = F.node_charge_density(self.node_charge, n_vol, spwt)
            self.potential, _, _ = fs.solve(self.node_charge, consts)
            m.c_ef[:] = F.electric_field(m.c2n, fs.c_sd, self.potential)
        self.last_remove, self.last_visits = rc, visits
        out = {"iter": self.iter, "size_before_move": n_before, "removed": rc, "size": self.size, "visits": visits}
        self.iter += 1
        return out

    def sort_now(self) -> bool:
        if self.fill == "Sort_All":
            return True
        if self.fill == "Sort_Periodic":
            return self.iter % self.fill_period == 0
        return False

    def finalize(self, remove_count: int) -> None:
        # opp_finalize_particle_move_core (opp_particle_organize_core.cpp:49-95)
        if remove_count <= 0:
            return
        dats = [self.pos, self.vel, self.lc, self.p2c]
        if self.sort_now():
            sort(self.size, self.m.n_cells, dats, 3)
        else:
            hole_fill(self.size, remove_count, self.p2c, dats)
        self.size -= remove_count

