"""Geometry evaluation on the grid (reference src/util.jl).

A geometry is a function of the grid coordinates, a boolean array of the grid's shape, or
(for sources and monitors) a tuple of coordinates meaning the nearest single grid point.
Functions are first evaluated on broadcast coordinate arrays (numpy semantics); a function
that cannot take arrays is evaluated point by point.  Linear cell indices are x fastest,
ix + Nx*(iy + Ny*iz), 0-based -- the column-major order of the reference's
CartesianIndex lists.
"""
import numpy as np


def _coords(grid, x=None, y=None, z=None):
    if grid.ndim == 1:
        return (grid.z if z is None else z,)
    if grid.ndim == 2:
        return (grid.x if x is None else x, grid.z if z is None else z)
    return (grid.x if x is None else x, grid.y if y is None else y, grid.z if z is None else z)


def geometry2bool(geometry, grid, coords=None):
    """``geometry2bool`` (util.jl:1-31): boolean array of the grid's shape."""
    shape = grid.shape
    if not callable(geometry):
        arr = np.asarray(geometry).astype(bool)
        if arr.shape != shape:
            raise ValueError(f"geometry array has shape {arr.shape}, grid has {shape}")
        return arr
    cs = coords if coords is not None else _coords(grid)
    nd = len(cs)
    open_cs = [np.asarray(c).reshape([-1 if k == j else 1 for k in range(nd)]) for j, c in enumerate(cs)]
    try:
        with np.errstate(all="ignore"):
            res = geometry(*open_cs)
        res = np.asarray(res)
        if res.dtype != bool and res.dtype.kind not in "iuf":
            raise TypeError
        return np.broadcast_to(res.astype(bool), shape).copy()
    except (ValueError, TypeError):
        out = np.zeros(shape, dtype=bool)
        for idx in np.ndindex(*shape):
            out[idx] = bool(geometry(*[float(cs[k][idx[k]]) for k in range(nd)]))
        return out


def linear_index(grid, idx):
    """0-based multi-index -> linear cell index, x fastest."""
    if grid.ndim == 1:
        return int(idx[0])
    if grid.ndim == 2:
        return int(idx[0]) + grid.Nx * int(idx[1])
    return int(idx[0]) + grid.Nx * (int(idx[1]) + grid.Ny * int(idx[2]))


def geometry2indices(geometry, grid, coords=None):
    """``geometry2indices`` (util.jl:35-100) as sorted 0-based linear cell indices."""
    cs = coords if coords is not None else _coords(grid)
    if isinstance(geometry, tuple):
        if len(geometry) != len(cs):
            raise ValueError("point geometry needs one coordinate per grid dimension")
        idx = [int(np.argmin(np.abs(np.asarray(c, dtype=np.float64) - g))) for c, g in zip(cs, geometry)]
        return np.array([linear_index(grid, idx)], dtype=np.int64)
    mask = geometry2bool(geometry, grid, cs)
    # the linear indices (x fastest) of the set cells, sorted: the row-major positions of the
    # set cells are converted, rather than making a column-major copy of the whole mask
    shape = tuple(grid.shape)
    pos = np.flatnonzero(np.ascontiguousarray(mask))
    idx = np.unravel_index(pos, shape)
    lin = np.zeros(len(pos), dtype=np.int64)
    stride = 1
    for k, n in enumerate(shape):
        lin += idx[k].astype(np.int64) * stride
        stride *= n
    lin.sort()
    return lin


def cell_coords(grid, cells, coords=None):
    """Coordinates (tuple of arrays) of linear cell indices."""
    cs = coords if coords is not None else _coords(grid)
    cells = np.asarray(cells, dtype=np.int64)
    if grid.ndim == 1:
        return (np.asarray(cs[0])[cells],)
    if grid.ndim == 2:
        ix, iz = cells % grid.Nx, cells // grid.Nx
        return (np.asarray(cs[0])[ix], np.asarray(cs[1])[iz])
    ix = cells % grid.Nx
    iy = (cells // grid.Nx) % grid.Ny
    iz = cells // (grid.Nx * grid.Ny)
    return (np.asarray(cs[0])[ix], np.asarray(cs[1])[iy], np.asarray(cs[2])[iz])


# ------------------------------------------------------------------------------------------
# Analytic shapes: geometries the library evaluates on the device (mfd_shape,
# include/maxwellfdtd.h).  Each is also a geometry function like the reference's closures:
# called with the grid coordinates it evaluates the same double-precision expression, in the
# same order, as the device does, so the map is the same whichever side builds it.  A 2-D
# grid's coordinates are (x, z) and a 1-D grid's z: the missing ones are 0, and a shape's
# points and vectors are given in the grid's own coordinates (2-D: (x, z); 1-D: (z,)).
# ------------------------------------------------------------------------------------------
def _to3(v, ndim):
    v = [float(a) for a in np.atleast_1d(v)]
    if len(v) == 3:
        return v
    if ndim == 2 and len(v) == 2:
        return [v[0], 0.0, v[1]]
    if ndim == 1 and len(v) == 1:
        return [0.0, 0.0, v[0]]
    raise ValueError("a shape's points and vectors need one value per grid dimension")


def _xyz(cs):
    z0 = np.zeros(1)
    if len(cs) == 3:
        return cs
    if len(cs) == 2:
        return cs[0], z0, cs[1]
    return z0, z0, cs[0]


class Shape:
    kind = 0

    def params(self, ndim):
        raise NotImplementedError

    def __call__(self, *cs):
        x, y, z = _xyz([np.asarray(c, dtype=np.float64) for c in cs])
        return self._covers(self.params(len(cs)), x, y, z)


class Ball(Shape):
    """((x-cx)^2 + (y-cy)^2) + (z-cz)^2 <= r^2."""
    kind = 1

    def __init__(self, center, radius):
        self.center, self.radius = center, float(radius)

    def params(self, ndim):
        return _to3(self.center, ndim) + [self.radius]

    @staticmethod
    def _covers(p, x, y, z):
        a, b, c = x - p[0], y - p[1], z - p[2]
        return (a * a + b * b) + c * c <= p[3] * p[3]


class Box(Shape):
    """lo <= (x, y, z) <= hi on every axis."""
    kind = 2

    def __init__(self, lo, hi):
        self.lo, self.hi = lo, hi

    def params(self, ndim):
        lo, hi = _to3(self.lo, ndim), _to3(self.hi, ndim)
        if ndim < 3:   # the missing axes are 0: the box spans them
            for k in ((1,) if ndim == 2 else (0, 1)):
                lo[k], hi[k] = -np.inf, np.inf
        return [lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]]

    @staticmethod
    def _covers(p, x, y, z):
        return (p[0] <= x) & (x <= p[1]) & (p[2] <= y) & (y <= p[3]) & (p[4] <= z) & (z <= p[5])


class Ellipsoid(Shape):
    """(((x-cx)/ax)^2 + ((y-cy)/ay)^2) + ((z-cz)/az)^2 <= 1."""
    kind = 3

    def __init__(self, center, semiaxes):
        self.center, self.semiaxes = center, semiaxes

    def params(self, ndim):
        ax = _to3(self.semiaxes, ndim)
        if ndim < 3:
            ax = [a if a != 0.0 else 1.0 for a in ax]   # a missing axis (coordinate 0, centre 0) adds 0
        return _to3(self.center, ndim) + ax

    @staticmethod
    def _covers(p, x, y, z):
        a, b, c = (x - p[0]) / p[3], (y - p[1]) / p[4], (z - p[2]) / p[5]
        return (a * a + b * b) + c * c <= 1.0


class Cylinder(Shape):
    """A circular cylinder along z: (x-cx)^2 + (y-cy)^2 <= r^2 and z0 <= z <= z1 (3-D)."""
    kind = 4

    def __init__(self, center_xy, radius, z0, z1):
        self.center_xy, self.radius, self.z0, self.z1 = center_xy, float(radius), float(z0), float(z1)

    def params(self, ndim):
        if ndim != 3:
            raise ValueError("Cylinder is a 3-D shape")
        cx, cy = (float(v) for v in self.center_xy)
        return [cx, cy, self.radius, self.z0, self.z1]

    @staticmethod
    def _covers(p, x, y, z):
        a, b = x - p[0], y - p[1]
        return (a * a + b * b <= p[2] * p[2]) & (p[3] <= z) & (z <= p[4])


class HalfSpace(Shape):
    """(nx x + ny y) + nz z >= d."""
    kind = 5

    def __init__(self, normal, d):
        self.normal, self.d = normal, float(d)

    def params(self, ndim):
        return _to3(self.normal, ndim) + [self.d]

    @staticmethod
    def _covers(p, x, y, z):
        return (p[0] * x + p[1] * y) + p[2] * z >= p[3]


class Everywhere(Shape):
    """Every cell (a whole-domain material)."""
    kind = 6

    def params(self, ndim):
        return []

    @staticmethod
    def _covers(p, x, y, z):
        return np.ones(np.broadcast_shapes(np.shape(x), np.shape(y), np.shape(z)), dtype=bool)
