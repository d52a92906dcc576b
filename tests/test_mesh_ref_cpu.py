"""The FemPIC box mesh pinned to the reference app's own mesh loader.

The compiled reference harness writes the box as the app's text mesh files and loads them
with load_mesh() (apps_codegen/app_fempic_cg/fempic_misc_mesh_loader.h ->
LoadVolumeMesh / LoadSurfaceMesh, apps/app_fempic/minifempic_funcs.h:230-583).  The
library's set-up (oppb_fempic_box_mesh, include/oppb_fempic.h) and the oracle's numpy
restatement (oracle/mesh.py) must give the same arrays bit for bit: node positions, volumes
and types, cell connectivity after the orientation flip, face neighbours, the alpha..delta
cofactors, cell volumes and centroids, and the inlet faces with their cells, edge vectors,
normals and areas.  The config meshes' coordinates survive the loader's mm conversion
exactly, so no tolerance is needed there.  On a box whose coordinates do not (spacings 0.14,
0.1, 0.1857...), the loader's positions differ from the library's by up to one ulp: the
integer arrays are still equal and the geometry agrees to 1e-15 of its magnitude.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mesh as OM
from oracle import ref_runner as R

pytestmark = pytest.mark.skipif(not R.available("seq"), reason="compiled reference (oracle/_ref) not built")

FIELDS = ("n_pos", "n_vol", "n_type", "c2n", "c2c", "c_det", "c_vol", "c_centroid", "if2c", "if2n", "if_u", "if_v",
          "if_norm", "if_area", "if_n_pos")
# config 1 / 3 (10x10x40 hexes, 24,000 tets), config 2 (48x48x192 hexes, 2,654,208 tets),
# a dyadic box and a box whose spacings are not representable and differ per axis.
EXACT = [(10, 10, 40, 1.0, 1.0, 4.0), (8, 8, 32, 1.0, 1.0, 4.0)]
ODD = (5, 3, 7, 0.7, 0.3, 1.3)
BOXES = EXACT + [ODD]
FULL = (48, 48, 192, 1.0, 1.0, 4.0)


def _bits(a: np.ndarray, dtype) -> np.ndarray:
    return np.ascontiguousarray(a).astype(dtype).view(np.uint8)


def _differing(ref: dict, mesh) -> list[str]:
    return [k for k in FIELDS if ref[k].shape != np.shape(getattr(mesh, k))
            or not np.array_equal(_bits(ref[k], ref[k].dtype), _bits(getattr(mesh, k), ref[k].dtype))]


@pytest.fixture(scope="module")
def ref_meshes():
    return {dims: R.box_mesh(dims) for dims in BOXES}


@pytest.mark.parametrize("dims", EXACT)
def test_library_mesh_equals_reference_loader(ref_meshes, dims):
    from oppb.fempic import HostMesh

    ref = ref_meshes[dims]
    hm = HostMesh(*dims, solve_field=False)
    assert (hm.n_nodes, hm.n_cells, hm.n_ifaces) == (ref["n_nodes"], ref["n_cells"], ref["n_ifaces"])
    assert _differing(ref, hm) == []


def test_library_mesh_matches_reference_loader_off_grid(ref_meshes):
    from oppb.fempic import HostMesh

    ref = ref_meshes[ODD]
    hm = HostMesh(*ODD, solve_field=False)
    assert "n_pos" in _differing(ref, hm)  # the case is the one meant: positions moved by the mm conversion
    for k in FIELDS:
        a, b = ref[k], getattr(hm, k)
        if a.dtype != np.float64:
            assert np.array_equal(a, b), k
        else:
            assert np.abs(a - b).max() <= 1e-15 * max(1.0, np.abs(a).max()), k


@pytest.mark.parametrize("dims", BOXES)
def test_oracle_mesh_equals_reference_loader(ref_meshes, dims):
    ref = ref_meshes[dims]
    assert _differing(ref, OM.box_mesh(*dims)) == []


def test_library_mesh_equals_reference_loader_fullsize():
    """The benchmark's 2,654,208-tet mesh (about 20 s: the loader's neighbour search)."""
    from oppb.fempic import HostMesh

    ref = R.box_mesh(FULL)
    assert _differing(ref, HostMesh(*FULL, solve_field=False)) == []


@pytest.mark.parametrize("dims,total", [(BOXES[0], 2000), (BOXES[2], 1000), (BOXES[0], 150)])
def test_injection_distribution_matches_library(dims, total):
    """The workload's distribution rule, as the reference harness and the oracle state it."""
    from oppb.fempic import HostMesh

    hm = HostMesh(*dims, solve_field=False)
    d = OM.area_distribution(hm.if_area, total)
    assert np.array_equal(d, hm.inject_distribution(total))
    assert d[-1] == total and np.all(np.diff(d) >= 0)
