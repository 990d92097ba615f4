"""Generate golden fixtures by running the reference's OWN functions on small meshes.

jNO cannot be imported in this image (``import jax`` fails; ``jno/bayesian.py:41`` needs equinox),
but the functions that fix the mesh, the P2 numbering, the boundary-facet set and the CSR pattern
are numpy code. This script parses them out of the reference sources with ``ast`` and executes
them with a numpy stand-in for ``jnp.asarray`` and a tiny ``meshio.Mesh`` record:

* ``Geometries.equi_distant_box``  -- jno/domain/geometries.py:203-300
* ``Geometries.equi_distant_rect`` -- jno/domain/geometries.py:44-200 (2-D triangles)
* ``_promote_to_degree``           -- jno/utils/solver/fem_utils.py:1979-2044
* ``compress_plan``                -- jno/utils/solver/fem_utils.py:4009-4060
* ``_boundary_facets``             -- jno/_fem.py:2695 (with ``_ref_interior_facet_dofs``
  jno/_fem.py:2635 and ``pack_face_keys`` jno/utils/solver/fem_facets.py:105-127)

The P2 reference interpolation points (what ``lagrange_interp_points(3, 2)`` returns from basix)
are the four vertices of the reference tet followed by the midpoints of the edges
``(2,3),(1,3),(1,2),(0,3),(0,2),(0,1)`` (``jno/utils/solver/fem_topology.py:44``); for the
triangle (``lagrange_interp_points(2, 2)``) the three vertices followed by the midpoints of the
edges ``(1,2),(0,2),(0,1)`` (``jno/utils/solver/fem_topology.py:36``).

Run from the repository root with the path of a jNO checkout:
    python tests/golden/make_golden.py <path to jNO>
Writes tests/golden/reference_small.npz (tetrahedra) and tests/golden/reference_small_2d.npz
(triangles). Nothing at test time reads the reference.
"""

import ast
import collections
import hashlib
import os
import sys
import typing

import numpy as np

REF = None  # the jNO checkout, set from the command line
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle.mesh import jitter_interior, jitter_interior_2d  # noqa: E402  (synthetic input only; not under test here)


class _StripRelativeImports(ast.NodeTransformer):
    def visit_ImportFrom(self, node):
        if node.level and node.level > 0:
            return ast.Pass()
        return node


def _extract(path, name, cls=None):
    src = open(os.path.join(REF, path)).read()
    tree = ast.parse(src)
    body = tree.body
    if cls is not None:
        body = next(n for n in tree.body if isinstance(n, ast.ClassDef) and n.name == cls).body
    fn = next(n for n in body if isinstance(n, ast.FunctionDef) and n.name == name)
    fn.decorator_list = []
    mod = ast.Module(body=[_StripRelativeImports().visit(fn)], type_ignores=[])
    ast.fix_missing_locations(mod)
    return compile(mod, f"{path}:{name}", "exec")


class _Mesh:
    def __init__(self, points, cells, cell_sets=None):
        self.points = points
        self.cells = cells
        self.cell_sets = cell_sets


class _JnpShim:
    @staticmethod
    def asarray(a, dtype=None):
        return np.asarray(a, dtype=dtype)


P2_REF = np.array(
    [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]
    + [
        [(a[0] + b[0]) / 2, (a[1] + b[1]) / 2, (a[2] + b[2]) / 2]
        for a, b in [
            (v[i], v[j])
            for v in [[[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]]
            for i, j in ((2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1))
        ]
    ],
    dtype=float,
)


P2_REF_TRI = np.array(
    [[0, 0], [1, 0], [0, 1]]
    + [
        [(a[0] + b[0]) / 2, (a[1] + b[1]) / 2]
        for a, b in [(v[i], v[j]) for v in [[[0, 0], [1, 0], [0, 1]]] for i, j in ((1, 2), (0, 2), (0, 1))]
    ],
    dtype=float,
)


def load_reference():
    g = {"np": np, "meshio": type("meshio", (), {"Mesh": _Mesh})}
    exec(_extract("jno/domain/geometries.py", "equi_distant_box", cls="Geometries"), g)
    exec(_extract("jno/domain/geometries.py", "equi_distant_rect", cls="Geometries"), g)
    ns = {
        "np": np,
        "jnp": _JnpShim,
        "_hashlib": hashlib,
        "_PLAN_CACHE": collections.OrderedDict(),
        "_PLAN_CACHE_MAX": 4,
        "List": typing.List,
        "Any": typing.Any,
        "Optional": typing.Optional,
    }
    exec(_extract("jno/utils/solver/fem_utils.py", "_promote_to_degree"), ns)
    exec(_extract("jno/utils/solver/fem_utils.py", "compress_plan"), ns)
    exec(_extract("jno/utils/solver/fem_facets.py", "pack_face_keys"), ns)
    ns["lagrange_interp_points"] = lambda dim, order, cell_type=None: P2_REF_TRI if dim == 2 else P2_REF
    exec(_extract("jno/_fem.py", "_ref_interior_facet_dofs"), ns)
    exec(_extract("jno/_fem.py", "_boundary_facets"), ns)
    return (g["equi_distant_box"], ns["_promote_to_degree"], ns["compress_plan"], ns["_boundary_facets"],
            g["equi_distant_rect"])


CASES = [(2, 2, 2), (3, 2, 4), (4, 4, 4)]
CASES_2D = [(2, 2), (3, 2), (5, 4)]


def _plan_and_facets(out, tag, plan, bfacets, dim, order, cells, ppts):
    T, nd = cells.shape
    rows = np.broadcast_to(cells[:, :, None], (T, nd, nd)).reshape(-1)
    cols = np.broadcast_to(cells[:, None, :], (T, nd, nd)).reshape(-1)
    idx, inverse, nse = plan(np.stack([rows, cols], axis=1).astype(np.int32))
    out[f"{tag}/p{order}_idx"] = np.asarray(idx)
    out[f"{tag}/p{order}_inverse"] = np.asarray(inverse)
    out[f"{tag}/p{order}_nse"] = np.array(nse)
    bf = bfacets(ppts, cells, dim, order)
    out[f"{tag}/p{order}_boundary"] = np.unique(np.asarray(bf).reshape(-1))


def main_2d(rect, promote, plan, bfacets):
    out = {}
    for nx, ny in CASES_2D:
        tag = f"{nx}x{ny}"
        mesh, dim, ds = rect(nx=nx, ny=ny, cell="triangle")(None)
        pts = np.asarray(mesh.points, dtype=float)[:, :dim]  # fem_native.py:250
        tris = np.asarray(mesh.cells[0][1], dtype=np.int64)
        out[f"{tag}/points"] = pts
        out[f"{tag}/tris"] = tris
        out[f"{tag}/ds"] = np.array(ds)
        jp = jitter_interior_2d(pts, nx, ny, seed=0)
        out[f"{tag}/jittered"] = jp
        p2_pts, p2_cells = promote(jp, tris, P2_REF_TRI)
        out[f"{tag}/p2_points"] = np.asarray(p2_pts)
        out[f"{tag}/p2_cells"] = np.asarray(p2_cells, dtype=np.int64)
        for order, cells, ppts in ((1, tris, jp), (2, np.asarray(p2_cells), np.asarray(p2_pts))):
            _plan_and_facets(out, tag, plan, bfacets, dim, order, cells, ppts)
    path = os.path.join(HERE, "reference_small_2d.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, sum(v.nbytes for v in out.values()), "bytes")


def main():
    box, promote, plan, bfacets, rect = load_reference()
    out = {}
    for nx, ny, nz in CASES:
        tag = f"{nx}x{ny}x{nz}"
        mesh, dim, ds = box(nx=nx, ny=ny, nz=nz, cell="tetra")(None)
        pts = np.asarray(mesh.points, dtype=float)
        tets = np.asarray(mesh.cells[0][1], dtype=np.int64)
        out[f"{tag}/points"] = pts
        out[f"{tag}/tets"] = tets
        out[f"{tag}/ds"] = np.array(ds)
        jp = jitter_interior(pts, nx, ny, nz, seed=0)
        out[f"{tag}/jittered"] = jp
        p2_pts, p2_cells = promote(jp, tets, P2_REF)
        out[f"{tag}/p2_points"] = np.asarray(p2_pts)
        out[f"{tag}/p2_cells"] = np.asarray(p2_cells, dtype=np.int64)
        for order, cells, ppts in ((1, tets, jp), (2, np.asarray(p2_cells), np.asarray(p2_pts))):
            _plan_and_facets(out, tag, plan, bfacets, 3, order, cells, ppts)
    path = os.path.join(HERE, "reference_small.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, sum(v.nbytes for v in out.values()), "bytes")
    main_2d(rect, promote, plan, bfacets)


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("reference", help="path of the jNO checkout whose functions are executed")
    REF = os.path.abspath(ap.parse_args().reference)
    main()
