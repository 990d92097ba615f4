"""Oracle: Kuhn box mesh, synthetic jitter, P2 promotion and boundary nodes (test infrastructure).

Restates, in vectorised numpy:
* ``Geometries.equi_distant_box(..., cell="tetra")`` -- ``jno/domain/geometries.py:203-300``:
  lattice points in C order ``idx = (i*(ny+1) + j)*(nz+1) + k`` (``:216``, ``:236-240``) and six
  Kuhn tets per voxel in (i, j, k, kuhn) order, corner bits ``(c>>2, c>>1, c)`` (``:242-258``).
* ``_promote_to_degree`` -- ``jno/utils/solver/fem_utils.py:1979-2044`` for a P2 simplex mesh:
  vertices keep ids ``0..nv-1``; every new node is numbered in first-encounter order over
  (cell, local dof), local dofs 4..9 being the edge midpoints on ``BASIX_TET_EDGES``
  (``jno/utils/solver/fem_topology.py:44``). The reference dedups by a coordinate hash; on a
  conforming mesh two midpoints coincide exactly when they are the same edge, so the edge key
  (min vertex, max vertex) is the same relation.
* ``_boundary_facets`` -- ``jno/_fem.py:2695``: a facet is boundary when exactly one cell has it;
  the Dirichlet set is every node on a boundary facet (P2: the facet's three edge midpoints too),
  as ``_boundary_node_ids`` (``jno/utils/solver/fem_native.py:2563-2636``) collects it.
* ``Geometries.equi_distant_rect(..., cell="triangle")`` -- ``jno/domain/geometries.py:44-100``:
  lattice points ``idx = i*(ny+1) + j`` (``:71-80``) and two triangles per rectangle,
  ``(p00, p10, p11)`` then ``(p00, p11, p01)`` in (i, j) order (``:85-98``); the 2-D path reads the
  points as ``[:, :2]`` (``jno/utils/solver/fem_native.py:250``). P2 triangles add their edge
  midpoints on ``BASIX_TRIANGLE_EDGES`` (``jno/utils/solver/fem_topology.py:36``); facets are edges.
"""

import numpy as np

#: Six Kuhn tets per voxel, local corner c encodes (di, dj, dk) = (c>>2 & 1, c>>1 & 1, c & 1).
KUHN = ((0, 4, 6, 7), (0, 4, 5, 7), (0, 2, 6, 7), (0, 2, 3, 7), (0, 1, 5, 7), (0, 1, 3, 7))
#: basix P2 tetrahedron edge order: local dof 4 + e sits on edge TET_EDGES[e].
TET_EDGES = ((2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1))
#: Facets of a tet as local vertex triples (the order of ``jno/_fem.py`` ``combos``).
TET_FACES = ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))
#: basix P2 triangle edge order: local dof 3 + e sits on edge TRI_EDGES[e].
TRI_EDGES = ((1, 2), (0, 2), (0, 1))
#: Facets (edges) of a triangle as local vertex pairs.
TRI_FACETS = ((0, 1), (0, 2), (1, 2))


def topology(nv):
    """(edges, facets) of a simplex with nv vertices (3: triangle, 4: tetrahedron)."""
    return (TRI_EDGES, TRI_FACETS) if nv == 3 else (TET_EDGES, TET_FACES)


def equi_distant_box(nx, ny, nz, x_range=(0.0, 1.0), y_range=(0.0, 1.0), z_range=(0.0, 1.0)):
    """Points f64[(nx+1)(ny+1)(nz+1), 3] and tets i64[6*nx*ny*nz, 4] of the structured Kuhn box."""
    X = np.linspace(x_range[0], x_range[1], nx + 1)
    Y = np.linspace(y_range[0], y_range[1], ny + 1)
    Z = np.linspace(z_range[0], z_range[1], nz + 1)
    xx, yy, zz = np.meshgrid(X, Y, Z, indexing="ij")
    points = np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])
    ny1, nz1 = ny + 1, nz + 1
    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    corner = np.stack(
        [((I + ((c >> 2) & 1)) * ny1 + (J + ((c >> 1) & 1))) * nz1 + (K + (c & 1)) for c in range(8)], axis=1
    )
    tets = corner[:, np.asarray(KUHN)].reshape(-1, 4).astype(np.int64)
    return points, tets


def jitter_interior(points, nx, ny, nz, seed, amp=0.1, x_range=(0.0, 1.0), y_range=(0.0, 1.0), z_range=(0.0, 1.0)):
    """Synthetic input: move every interior lattice vertex by U(-amp*h, amp*h) per axis.

    Interior means lattice index strictly inside on all three axes; boundary vertices are untouched.
    The draw is ``np.random.default_rng(seed).uniform(-amp, amp, (n_interior, 3)) * h`` in node-id
    order, h = (hx, hy, hz) the lattice spacing.
    """
    pts = np.array(points, dtype=np.float64, copy=True)
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    inner = ((i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)).ravel()
    h = np.array(
        [(x_range[1] - x_range[0]) / nx, (y_range[1] - y_range[0]) / ny, (z_range[1] - z_range[0]) / nz]
    )
    rng = np.random.default_rng(seed)
    d = rng.uniform(-amp, amp, size=(int(inner.sum()), 3)) * h[None, :]
    pts[inner] += d
    return pts


def equi_distant_rect(nx, ny, x_range=(0.0, 1.0), y_range=(0.0, 1.0)):
    """Points f64[(nx+1)(ny+1), 2] and triangles i64[2*nx*ny, 3] of the structured rectangle."""
    X = np.linspace(x_range[0], x_range[1], nx + 1)
    Y = np.linspace(y_range[0], y_range[1], ny + 1)
    xx, yy = np.meshgrid(X, Y, indexing="ij")
    points = np.column_stack([xx.ravel(), yy.ravel()])
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    I, J = I.ravel(), J.ravel()
    p0 = I * (ny + 1) + J
    p1 = (I + 1) * (ny + 1) + J
    p2 = (I + 1) * (ny + 1) + J + 1
    p3 = I * (ny + 1) + J + 1
    tris = np.stack([np.stack([p0, p1, p2], axis=1), np.stack([p0, p2, p3], axis=1)], axis=1)
    return points, tris.reshape(-1, 3).astype(np.int64)


def jitter_interior_2d(points, nx, ny, seed, amp=0.1, x_range=(0.0, 1.0), y_range=(0.0, 1.0)):
    """Synthetic input: ``jitter_interior`` on the rectangle lattice (interior on both axes)."""
    pts = np.array(points, dtype=np.float64, copy=True)
    i, j = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    inner = ((i > 0) & (i < nx) & (j > 0) & (j < ny)).ravel()
    h = np.array([(x_range[1] - x_range[0]) / nx, (y_range[1] - y_range[0]) / ny])
    rng = np.random.default_rng(seed)
    pts[inner] += rng.uniform(-amp, amp, size=(int(inner.sum()), 2)) * h[None, :]
    return pts


def promote_p2(points, tets):
    """P2 node mesh: (points_p2 f64[n,dim], cells_p2 i64[T,nd]) in basix dof order (nd = 10 / 6)."""
    points = np.asarray(points, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    nv = points.shape[0]
    edges, _ = topology(tets.shape[1])
    ea = tets[:, [e[0] for e in edges]]
    eb = tets[:, [e[1] for e in edges]]
    lo, hi = np.minimum(ea, eb).ravel(), np.maximum(ea, eb).ravel()
    key = lo * nv + hi
    _, first, inverse = np.unique(key, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    edge_id = nv + rank[inverse.reshape(-1)]
    cells = np.concatenate([tets, edge_id.reshape(-1, len(edges))], axis=1)
    fa, fb = ea.ravel()[first[order]], eb.ravel()[first[order]]
    mid = 0.5 * points[fa] + 0.5 * points[fb]
    return np.concatenate([points, mid], axis=0), cells


def boundary_nodes(cells, order, nv=4):
    """Sorted unique node ids on boundary facets (facets owned by exactly one cell); nv = 4
    (tetrahedra: facets are faces) or 3 (triangles: facets are edges)."""
    cells = np.asarray(cells, dtype=np.int64)
    edges, facets = topology(nv)
    verts = cells[:, :nv]
    faces = np.concatenate([verts[:, list(f)] for f in facets], axis=0)
    canon = np.sort(faces, axis=1)
    n = int(canon.max()) + 1
    keys = canon[:, 0]
    for k in range(1, canon.shape[1]):
        keys = keys * n + canon[:, k]
    _, idx, counts = np.unique(keys, return_index=True, return_counts=True)
    bidx = idx[counts == 1]
    nodes = [faces[bidx].reshape(-1)]
    if order == 2:
        ncell = cells.shape[0]
        face_of, cell_of = bidx // ncell, bidx % ncell
        for fi, f in enumerate(facets):
            sel = cell_of[face_of == fi]
            for e, (a, b) in enumerate(edges):
                if a in f and b in f:
                    nodes.append(cells[sel, nv + e])
    return np.unique(np.concatenate(nodes))


def kuhn_cube(n, order=1, seed=0, amp=0.1):
    """The synthetic workload mesh: unit cube, n^3 hexes x 6 Kuhn tets, interior jitter from ``seed``.

    Returns ``(points_f, cells_f, tets_p1, points_p1)``; for P1 the first pair equals the last.
    """
    pts, tets = equi_distant_box(n, n, n)
    pts = jitter_interior(pts, n, n, n, seed, amp)
    if order == 1:
        return pts, tets, tets, pts
    pf, cf = promote_p2(pts, tets)
    return pf, cf, tets, pts


def unit_square(n, order=1, seed=0, amp=0.1):
    """The 2-D synthetic mesh: unit square, n^2 rectangles x 2 triangles, interior jitter from ``seed``.

    Returns ``(points_f, cells_f, tris_p1, points_p1)`` with 2 coordinates per point.
    """
    pts, tris = equi_distant_rect(n, n)
    pts = jitter_interior_2d(pts, n, n, seed, amp)
    if order == 1:
        return pts, tris, tris, pts
    pf, cf = promote_p2(pts, tris)
    return pf, cf, tris, pts


def logk_field(ntet, seed, sigma=0.5):
    """Per-element log-conductivity: ``default_rng(seed).normal(0, sigma, ntet)``."""
    return np.random.default_rng(seed).normal(0.0, sigma, ntet)
