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
