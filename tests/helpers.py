"""Shared set-up of the tests: cached meshes and seeded particle states."""
from __future__ import annotations

import functools

import numpy as np

from oppb.fempic import HostMesh

REMOVED = 2147483647


@functools.lru_cache(maxsize=None)
def mesh(nx: int = 10, ny: int = 10, nz: int = 40, lx: float = 1.0, ly: float = 1.0, lz: float = 4.0) -> HostMesh:
    """Box mesh; the default is the 10x10x40-hex, 24,000-tet case."""
    return HostMesh(nx, ny, nz, lx, ly, lz)


def random_particles(hm: HostMesh, n: int, seed: int, spread: float = 0.05, far_frac: float = 0.05,
                     outside_frac: float = 0.02):
    """Particles placed near a random cell's centroid (displacement ~ spread), a fraction
    started in a cell far from their position (long walks), a fraction outside the box
    (removals).  Returns AoS pos [n,3] and p2c [n]."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(0, hm.n_cells, n).astype(np.int32)
    pos = hm.c_centroid[cells] + rng.normal(0.0, spread, (n, 3))
    lo = np.zeros(3)
    hi = np.array(hm.dims[3:6])
    far = rng.random(n) < far_frac
    cells[far] = rng.integers(0, hm.n_cells, far.sum())
    out = rng.random(n) < outside_frac
    pos[out] = lo + (hi - lo) * rng.random((out.sum(), 3)) + np.where(rng.random((out.sum(), 3)) < 0.5, -1, 1) * 0.3
    # Particles exactly on cell faces / vertices: ties in the argmin and lambda == 0.
    on = rng.random(n) < 0.01
    pos[on] = hm.n_pos[hm.c2n[cells[on], 0]]
    return np.ascontiguousarray(pos), cells


def advec_edge_particles(m, ppc: int, v_sd: float, seed: int):
    """NESO-advection particles (oppb.advec.particles) with a quarter resting on their cell's
    lower x edge and a quarter on its lower y edge: points two cells share, where the walk's
    start cell (the direct-hop seed or the previous cell) decides the final one.  Returns AoS
    pos, vel, mdir, p2c."""
    from oppb.advec import particles

    pos, vel, mdir, p2c = particles(m, ppc, v_sd, seed)
    rng = np.random.default_rng(seed + 1)
    ia = rng.choice(len(p2c), len(p2c) // 4, replace=False)
    ib = rng.choice(len(p2c), len(p2c) // 4, replace=False)
    pos[ia, 0] = m.c_pos_ll[p2c[ia], 0]
    pos[ib, 1] = m.c_pos_ll[p2c[ib], 1]
    vel[ia] = 0.0
    vel[ib] = 0.0
    return pos, vel, mdir, p2c
