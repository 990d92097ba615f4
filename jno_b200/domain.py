"""Mesh front end: the structured Kuhn box, the triangulated rectangle and a ``jno.domain``-shaped
holder (host, numpy).

``equi_distant_box`` follows ``Geometries.equi_distant_box(..., cell="tetra")``
(jno/domain/geometries.py:203-300): lattice points in C order ``idx = (i(ny+1) + j)(nz+1) + k`` and
six Kuhn tets per voxel in (i, j, k, kuhn) order, corner bits ``(c>>2, c>>1, c)``.
``equi_distant_rect`` follows ``Geometries.equi_distant_rect(..., cell="triangle")``
(jno/domain/geometries.py:44-200): lattice points ``idx = i(ny+1) + j`` with z = 0 and two
triangles ``(p00, p10, p11)``, ``(p00, p11, p01)`` per rectangle in (i, j) order. Both return a
``constructor(geo) -> (mesh, dim, ds)`` like the reference; ``domain(constructor)`` builds the mesh,
and the FEM reads its points as ``[:, :dim]`` (jno/utils/solver/fem_native.py:250).
"""

import numpy as np

KUHN = ((0, 4, 6, 7), (0, 4, 5, 7), (0, 2, 6, 7), (0, 2, 3, 7), (0, 1, 5, 7), (0, 1, 3, 7))


class Mesh:
    """Minimal mesh record: ``points`` f64[nv, 3] and the simplex cells i64[T, dim+1]
    (``tetra`` for dim 3, ``triangle`` for dim 2; a 2-D mesh has z = 0)."""

    def __init__(self, points, tets, dim=3):
        self.points = np.asarray(points, dtype=np.float64)
        self.dim = dim
        self.tets = np.asarray(tets, dtype=np.int64)  # the cells (tetrahedra, or triangles in 2-D)
        self.cells_dict = {"tetra" if dim == 3 else "triangle": self.tets}


def box_points_tets(nx, ny, nz, x_range=(0.0, 1.0), y_range=(0.0, 1.0), z_range=(0.0, 1.0)):
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


def equi_distant_box(x_range=(0, 1), y_range=(0, 1), z_range=(0, 1), nx=8, ny=8, nz=8, cell="tetra"):
    """Structured Kuhn-tet box constructor (the reference's ``equi_distant_box`` contract)."""
    if cell != "tetra":
        raise NotImplementedError("only cell='tetra' is on the B200 path (hexahedra are out of scope)")

    def constructor(geo=None):
        pts, tets = box_points_tets(nx, ny, nz, x_range, y_range, z_range)
        ds = min((x_range[1] - x_range[0]) / nx, (y_range[1] - y_range[0]) / ny, (z_range[1] - z_range[0]) / nz)
        return Mesh(pts, tets), 3, ds

    constructor.lattice = (nx, ny, nz, x_range, y_range, z_range)
    return constructor


def rect_points_tris(nx, ny, x_range=(0.0, 1.0), y_range=(0.0, 1.0)):
    X = np.linspace(x_range[0], x_range[1], nx + 1)
    Y = np.linspace(y_range[0], y_range[1], ny + 1)
    xx, yy = np.meshgrid(X, Y, indexing="ij")
    points = np.column_stack([xx.ravel(), yy.ravel(), np.zeros((nx + 1) * (ny + 1))])
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    I, J = I.ravel(), J.ravel()
    p00, p10 = I * (ny + 1) + J, (I + 1) * (ny + 1) + J
    p11, p01 = p10 + 1, p00 + 1
    tris = np.stack([np.stack([p00, p10, p11], 1), np.stack([p00, p11, p01], 1)], axis=1)
    return points, tris.reshape(-1, 3).astype(np.int64)


def equi_distant_rect(x_range=(0, 1), y_range=(0, 1), nx=10, ny=10, cell="triangle"):
    """Structured triangulated rectangle constructor (the reference's ``equi_distant_rect`` contract)."""
    if cell != "triangle":
        raise NotImplementedError("only cell='triangle' is on the B200 path (quadrilaterals are out of scope)")

    def constructor(geo=None):
        pts, tris = rect_points_tris(nx, ny, x_range, y_range)
        ds = min((x_range[1] - x_range[0]) / nx, (y_range[1] - y_range[0]) / ny)
        return Mesh(pts, tris, dim=2), 2, ds

    constructor.lattice = (nx, ny, x_range, y_range)
    return constructor


def jitter_interior_2d(points, nx, ny, seed, amp=0.1, x_range=(0.0, 1.0), y_range=(0.0, 1.0)):
    """``jitter_interior`` on the rectangle lattice: ``default_rng(seed).uniform(-amp, amp,
    (n_interior, 2)) * h`` moves the interior vertices in x and y (z stays 0)."""
    pts = np.array(points, dtype=np.float64, copy=True)
    i, j = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    inner = ((i > 0) & (i < nx) & (j > 0) & (j < ny)).ravel()
    h = np.array([(x_range[1] - x_range[0]) / nx, (y_range[1] - y_range[0]) / ny])
    rng = np.random.default_rng(seed)
    pts[inner, :2] += rng.uniform(-amp, amp, size=(int(inner.sum()), 2)) * h[None, :]
    return pts


def jitter_interior(points, nx, ny, nz, seed, amp=0.1, x_range=(0.0, 1.0), y_range=(0.0, 1.0), z_range=(0.0, 1.0)):
    """Synthetic workload input: move every interior lattice vertex by U(-amp h, amp h) per axis.

    ``np.random.default_rng(seed).uniform(-amp, amp, (n_interior, 3)) * h`` in node-id order.
    """
    pts = np.array(points, dtype=np.float64, copy=True)
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    inner = ((i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)).ravel()
    h = np.array([(x_range[1] - x_range[0]) / nx, (y_range[1] - y_range[0]) / ny, (z_range[1] - z_range[0]) / nz])
    rng = np.random.default_rng(seed)
    pts[inner] += rng.uniform(-amp, amp, size=(int(inner.sum()), 3)) * h[None, :]
    return pts


class domain:
    """``jno.domain(constructor)``: holds the built mesh and hands out FEM symbols."""

    def __init__(self, constructor, jitter=None, seed=0, time=None):
        """``time=(t0, t1, n_steps)`` makes the domain transient: the time grid has n_steps points,
        dt = (t1 - t0) / (n_steps - 1) (jno/utils/solver/time_route.py:32-58)."""
        mesh, dim, ds = constructor(None)
        self.time = None if time is None else (float(time[0]), float(time[1]), int(time[2]))
        if dim not in (2, 3):
            raise NotImplementedError("only 2-D triangle and 3-D tetrahedral meshes are on the B200 path")
        self.built_mesh = mesh
        self.dimension = dim
        self.ds = ds
        if jitter:
            if dim == 3:
                nx, ny, nz, xr, yr, zr = constructor.lattice
                mesh.points = jitter_interior(mesh.points, nx, ny, nz, seed, jitter, xr, yr, zr)
            else:
                nx, ny, xr, yr = constructor.lattice
                mesh.points = jitter_interior_2d(mesh.points, nx, ny, seed, jitter, xr, yr)

    @classmethod
    def from_mesh(cls, points, tets):
        """A domain over given cells: tetrahedra i64[T, 4], or triangles i64[T, 3] (2-D)."""
        obj = cls.__new__(cls)
        dim = int(np.asarray(tets).shape[1]) - 1
        pts = np.asarray(points, dtype=np.float64)
        if pts.shape[1] == 2:
            pts = np.column_stack([pts, np.zeros(pts.shape[0])])
        obj.built_mesh = Mesh(pts, tets, dim=dim)
        obj.dimension = dim
        obj.ds = None
        obj.time = None
        return obj

    def _cells_p1(self):
        return self.built_mesh.tets

    def fem_symbols(self, names=("u", "v"), order=1, space=None, value_shape=None):
        from .trace import FieldSymbol

        if value_shape not in (None, (), 1):
            raise NotImplementedError("vector-valued fields are outside the B200 scalar Poisson path")
        if space == "P0":
            return (FieldSymbol(names[0], "trial", self, 0, "P0"), FieldSymbol(names[1], "test", self, 0, "P0"))
        if order not in (1, 2):
            raise NotImplementedError("only Lagrange P1/P2 are on the B200 path")
        return (FieldSymbol(names[0], "trial", self, order), FieldSymbol(names[1], "test", self, order))

    def variable(self, region, split=True):
        from .trace import Coordinate

        if region not in ("interior", "boundary", "initial"):
            raise NotImplementedError(
                f"region {region!r}: only 'interior', 'boundary' and 'initial' are on the B200 path")
        if region == "initial" and self.time is None:
            raise ValueError("the 'initial' region needs a transient domain (domain(..., time=(t0, t1, n_steps)))")
        coords = tuple(Coordinate(region, a) for a in range(self.dimension))
        return coords + (Coordinate(region, "t"),) if self.time is not None else coords
