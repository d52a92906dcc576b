"""TEST INFRASTRUCTURE ONLY — the FemPIC box mesh restated in numpy from the app's mesh
loader, for the oracle and the CPU-baseline port.

The box is the workload's: nx*ny*nz hexahedra, node i + (nx+1)(j + (ny+1)k) at
(i hx, j hy, k hz) (the last node of an axis at the box length), hexahedron (i,j,k) cut into
6 tetrahedra along its main diagonal, tetrahedron t walking 000 -> e_a -> e_a + e_b -> 111 for
the t-th permutation (a,b,c) of the axes; the inlet is the two triangles (000, 110, 100) and
(000, 010, 110) of every z=0 hexahedron face, the wall the z=lz nodes.  The geometry follows
apps/app_fempic/minifempic_funcs.h, operation by operation:
  volume (1/6) det4 and the ABCD -> ADBC flip                      :284-313
  alpha..delta cofactors per vertex                                  :316-382
  face neighbours (the tetrahedron sharing the face opposite v)      :386-437
  node volumes from the centroid's weights, OPEN nodes               :440-474 (XtoLtet :199-211)
  inlet cell, u, v, unit normal and area (no inversion)              :508-583
INLET and FIXED node types come from the inlet and wall surfaces (:488-505).  numpy applies
one rounding per elementwise operation, so every value equals the loader's C++ (compiled
without FMA contraction); tests/test_mesh_ref_cpu.py checks it against the compiled loader.
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np

NORMAL, OPEN, INLET, FIXED = 0, 1, 2, 3
_PERM = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
_COF = ((1, 2, 3), (3, 2, 0), (3, 0, 1), (1, 0, 2))  # v2, v3, v4 of vertex v (minifempic_funcs.h:323-330)
_FACE = ((1, 2, 3), (2, 3, 0), (3, 0, 1), (0, 1, 2))  # vertices of the face opposite v (:397-402)


def _det3(a, b, c):
    """det3 of rows a, b, c (each [..., 3]), first-row cofactor expansion (minifempic_funcs.h:69-73)."""
    return (a[..., 0] * (b[..., 1] * c[..., 2] - b[..., 2] * c[..., 1])
            - a[..., 1] * (b[..., 0] * c[..., 2] - b[..., 2] * c[..., 0])
            + a[..., 2] * (b[..., 0] * c[..., 1] - b[..., 1] * c[..., 0]))


def _det4_ones(p):
    """det4 of [[1, p_v]] for v = 0..3 (p [n, 4, 3]), first-row expansion (minifempic_funcs.h:75-103)."""
    one = np.ones(p.shape[0])

    def rows(cols):  # rows 1..3 of M restricted to the given columns
        m = np.concatenate([one[:, None, None].repeat(3, axis=1), p[:, 1:, :]], axis=2)  # [n, 3, 4]
        return [m[:, r, list(cols)] for r in range(3)]

    m0, m1, m2, m3 = rows((1, 2, 3)), rows((0, 2, 3)), rows((0, 1, 3)), rows((0, 1, 2))
    return (one * _det3(*m0) - p[:, 0, 0] * _det3(*m1) + p[:, 0, 1] * _det3(*m2) - p[:, 0, 2] * _det3(*m3))


def box_nodes(nx, ny, nz, lx, ly, lz):
    """Node positions as the loader reads them: mm values in the file, divided by 1000."""
    def axis(n, l):
        h = l / n
        x = np.arange(n + 1, dtype=np.float64) * h
        x[n] = l
        return (x * 1000.0) / 1000.0

    z, y, x = np.meshgrid(axis(nz, lz), axis(ny, ly), axis(nx, lx), indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)


def box_mesh(nx, ny, nz, lx, ly, lz):
    NX, NY = nx + 1, ny + 1
    n_pos = box_nodes(nx, ny, nz, lx, ly, lz)
    nid = lambda i, j, k: i + NX * (j + NY * k)  # noqa: E731
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    tets = []
    for a, b, _ in _PERM:
        o1 = np.zeros((3,), int)
        o1[a] = 1
        o2 = o1.copy()
        o2[b] = 1
        tets.append(np.stack([nid(i, j, k), nid(i + o1[0], j + o1[1], k + o1[2]),
                              nid(i + o2[0], j + o2[1], k + o2[2]), nid(i + 1, j + 1, k + 1)], axis=1))
    c2n = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int32)
    nc = len(c2n)

    # Volumes, with the ABCD -> ADBC flip where negative.
    vol = (1.0 / 6.0) * _det4_ones(n_pos[c2n])
    neg = vol < 0
    c2n[neg, 1], c2n[neg, 3] = c2n[neg, 3].copy(), c2n[neg, 1].copy()
    vol = np.where(neg, -vol, vol)
    p = n_pos[c2n]  # [nc, 4, 3]
    one = np.ones(nc)
    c_det = np.empty((nc, 4, 4))
    for v, (v2, v3, v4) in enumerate(_COF):
        a, b, c = p[:, v2], p[:, v3], p[:, v4]
        c_det[:, v, 0] = _det3(a, b, c)
        sel = lambda q, d0, d1: np.stack([one, q[:, d0], q[:, d1]], axis=1)  # noqa: E731
        c_det[:, v, 1] = _det3(sel(a, 1, 2), sel(b, 1, 2), sel(c, 1, 2))
        c_det[:, v, 2] = _det3(sel(a, 0, 2), sel(b, 0, 2), sel(c, 0, 2))
        c_det[:, v, 3] = _det3(sel(a, 0, 1), sel(b, 0, 1), sel(c, 0, 1))

    # Face neighbours: the other tetrahedron holding the three vertices of the face opposite v.
    faces = np.sort(np.stack([c2n[:, list(f)] for f in _FACE], axis=1), axis=2).reshape(-1, 3).astype(np.int64)
    key = (faces[:, 0] << 42) | (faces[:, 1] << 21) | faces[:, 2]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    same = np.flatnonzero(ks[1:] == ks[:-1])
    c2c = np.full(4 * nc, -1, np.int32)
    c2c[order[same]] = order[same + 1] // 4
    c2c[order[same + 1]] = order[same] // 4
    c2c = c2c.reshape(nc, 4)

    # Node volumes: lc of the centroid times the cell volume, in cell order; OPEN nodes.
    cen = np.zeros((nc, 3))
    for v in range(4):
        cen = cen + 0.25 * p[:, v]
    lc = np.stack([(1.0 / 6.0) * (c_det[:, v, 0] - cen[:, 0] * c_det[:, v, 1] + cen[:, 1] * c_det[:, v, 2]
                                  - cen[:, 2] * c_det[:, v, 3]) / vol for v in range(4)], axis=1)
    n_vol = np.zeros(len(n_pos))
    np.add.at(n_vol, c2n.ravel(), (lc * vol[:, None]).ravel())
    n_type = np.zeros(len(n_pos), np.int32)
    for v in range(4):
        open_face = c2c[:, v] < 0
        for q in range(4):
            if q != v:
                n_type[c2n[open_face, q]] = OPEN
    n_type[nid(np.arange(NX)[None, :], np.arange(NY)[:, None], 0).ravel()] = INLET
    n_type[nid(np.arange(NX)[None, :], np.arange(NY)[:, None], nz).ravel()] = FIXED

    # Inlet triangles, their cell (the tetrahedron holding all three nodes), u, v, normal, area.
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()
    n000, n100, n010, n110 = nid(ii, jj, 0), nid(ii + 1, jj, 0), nid(ii, jj + 1, 0), nid(ii + 1, jj + 1, 0)
    if2n = np.stack([np.stack([n000, n110, n100], 1), np.stack([n000, n010, n110], 1)], axis=1).reshape(-1, 3)
    tri_key = np.sort(if2n, axis=1).astype(np.int64)
    tri_key = (tri_key[:, 0] << 42) | (tri_key[:, 1] << 21) | tri_key[:, 2]
    pos_in = np.searchsorted(ks, tri_key)
    if2c = (order[pos_in] // 4).astype(np.int32)
    p1, p2, p3 = n_pos[if2n[:, 0]], n_pos[if2n[:, 1]], n_pos[if2n[:, 2]]
    u, w = p2 - p1, p3 - p1
    nrm = np.stack([u[:, 2] * w[:, 1] - u[:, 1] * w[:, 2], u[:, 0] * w[:, 2] - u[:, 2] * w[:, 0],
                    u[:, 1] * w[:, 0] - u[:, 0] * w[:, 1]], axis=1)
    ln = np.sqrt(nrm[:, 0] * nrm[:, 0] + nrm[:, 1] * nrm[:, 1] + nrm[:, 2] * nrm[:, 2])
    return SimpleNamespace(
        n_nodes=len(n_pos), n_cells=nc, n_ifaces=len(if2n), n_pos=n_pos, n_vol=n_vol, n_type=n_type,
        c2n=c2n, c2c=c2c, c_det=c_det.reshape(nc, 16), c_vol=vol, c_centroid=cen, if2c=if2c,
        if2n=if2n.astype(np.int32), if_u=u, if_v=w, if_norm=nrm / ln[:, None], if_area=ln / 2,
        if_n_pos=np.concatenate([p1, p2, p3], axis=1), c_ef=np.zeros((nc, 3)))


def static_field(mesh, phi_inlet: float, phi_fixed: float, lz: float) -> np.ndarray:
    """The cell field of the workload's Laplace problem (phi_inlet at z=0, phi_fixed at z=lz,
    natural boundary elsewhere): its exact discrete solution is linear in z, so every cell's
    field is (0, 0, (phi_inlet - phi_fixed) / lz)."""
    ef = np.zeros((mesh.n_cells, 3))
    ef[:, 2] = (phi_inlet - phi_fixed) / lz
    return ef


def area_distribution(if_area: np.ndarray, total: int) -> np.ndarray:
    """The workload's injection distribution: cumulative counts per inlet face from the
    rounded cumulative area share, the last face closing at `total` (sequential sums)."""
    n = len(if_area)
    area = 0.0
    for a in if_area:
        area += float(a)
    dist = np.zeros(n, np.int32)
    acc = 0.0
    for f in range(n):
        acc += float(if_area[f])
        x = float(total) * (acc / area)
        r = math.floor(x)
        cum = total if f == n - 1 else int(r) + (1 if x - r >= 0.5 else 0)  # llround: halves away from 0
        dist[f] = min(cum, total)
    return np.maximum.accumulate(dist)


def write_box_files(dims, out_dir) -> dict:
    """The box as the app's text mesh files (the formats LoadVolumeMesh and LoadSurfaceMesh
    read, apps/app_fempic/minifempic_funcs.h:230-270,477-520), the same text the reference
    harness writes: mesh.dat (node list in mm, 304 tetrahedra), inlet.dat (the z=0 nodes and the
    203 inlet triangles), wall.dat (the z=lz nodes).  Returns the three paths."""
    from pathlib import Path

    nx, ny, nz, lx, ly, lz = dims
    out = Path(out_dir)
    NX, NY = nx + 1, ny + 1

    def coords(n, l):
        h = l / n
        x = [float(i) * h for i in range(n + 1)]
        x[n] = l
        return [repr(v * 1000.0) for v in x]

    cx, cy, cz = coords(nx, lx), coords(ny, ly), coords(nz, lz)
    nid = lambda i, j, k: i + NX * (j + NY * k) + 1  # noqa: E731
    node = lambda i, j, k: f"{nid(i, j, k)} {cx[i]} {cy[j]} {cz[k]}"  # noqa: E731
    lines = [f"{NX * NY * (nz + 1)} {6 * nx * ny * nz}"]
    lines += [node(i, j, k) for k in range(nz + 1) for j in range(NY) for i in range(NX)]
    e = 1
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for a, b, _ in _PERM:
                    o1 = [0, 0, 0]
                    o1[a] = 1
                    o2 = list(o1)
                    o2[b] = 1
                    lines.append(f"{e} 304 {nid(i, j, k)} {nid(i + o1[0], j + o1[1], k + o1[2])} "
                                 f"{nid(i + o2[0], j + o2[1], k + o2[2])} {nid(i + 1, j + 1, k + 1)}")
                    e += 1
    (out / "mesh.dat").write_text("\n".join(lines) + "\n")
    lines = [f"{NX * NY} {2 * nx * ny}"] + [node(i, j, 0) for j in range(NY) for i in range(NX)]
    e = 1
    for j in range(ny):
        for i in range(nx):
            n000, n100, n010, n110 = nid(i, j, 0), nid(i + 1, j, 0), nid(i, j + 1, 0), nid(i + 1, j + 1, 0)
            lines += [f"{e} 203 {n000} {n110} {n100}", f"{e + 1} 203 {n000} {n010} {n110}"]
            e += 2
    (out / "inlet.dat").write_text("\n".join(lines) + "\n")
    lines = [f"{NX * NY} 0"] + [node(i, j, nz) for j in range(NY) for i in range(NX)]
    (out / "wall.dat").write_text("\n".join(lines) + "\n")
    return {"global_mesh": out / "mesh.dat", "inlet_mesh": out / "inlet.dat", "wall_mesh": out / "wall.dat"}
