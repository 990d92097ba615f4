"""The product's host mesh front end (``jno_b200.domain``) against the fixtures made by running the
reference's own ``Geometries.equi_distant_box`` / ``equi_distant_rect`` (jno/domain/geometries.py:
203-300, 44-200): lattice points, Kuhn tets / triangles in the reference's order, the cell size ``ds``
and the seeded interior jitter the parity tests feed both sides. Bit-exact: this is index and
coordinate layout, not arithmetic."""

import importlib

import numpy as np
import pytest

dm = importlib.import_module("jno_b200.domain")  # the module (the package exports its `domain` class)

CASES = [(2, 2, 2), (3, 2, 4), (4, 4, 4)]
CASES_2D = [(2, 2), (3, 2), (5, 4)]


@pytest.mark.parametrize("nx,ny,nz", CASES)
def test_box_matches_reference_fixture(golden, nx, ny, nz):
    tag = f"{nx}x{ny}x{nz}"
    pts, tets = dm.box_points_tets(nx, ny, nz)
    assert np.array_equal(pts, golden[f"{tag}/points"])
    assert np.array_equal(tets, golden[f"{tag}/tets"])
    mesh, dim, ds = dm.equi_distant_box(nx=nx, ny=ny, nz=nz)(None)
    assert dim == 3 and ds == float(golden[f"{tag}/ds"])
    assert np.array_equal(mesh.points, golden[f"{tag}/points"]) and np.array_equal(mesh.tets, golden[f"{tag}/tets"])
    assert np.array_equal(dm.jitter_interior(pts, nx, ny, nz, seed=0), golden[f"{tag}/jittered"])


@pytest.mark.parametrize("nx,ny", CASES_2D)
def test_rect_matches_reference_fixture(golden2d, nx, ny):
    tag = f"{nx}x{ny}"
    pts, tris = dm.rect_points_tris(nx, ny)
    assert np.array_equal(pts[:, :2], golden2d[f"{tag}/points"])
    assert np.array_equal(tris, golden2d[f"{tag}/tris"])
    mesh, dim, ds = dm.equi_distant_rect(nx=nx, ny=ny)(None)
    assert dim == 2 and ds == float(golden2d[f"{tag}/ds"])
    assert np.array_equal(mesh.points[:, :2], golden2d[f"{tag}/points"])
    assert np.array_equal(dm.jitter_interior_2d(pts, nx, ny, seed=0)[:, :2], golden2d[f"{tag}/jittered"])
