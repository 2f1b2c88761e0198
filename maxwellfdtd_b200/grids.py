"""Grids (reference src/grids.jl).

Coordinates follow Julia's ``range(start, stop, length)`` for Float64 end points: when the
end points are decimal literals Julia finds their exact rational values (``Base.rat``) and
returns correctly rounded points of the exact linear range, so e.g. ``z == 0`` holds on a
grid from -2e-6 to 72e-6.  This module computes the same points from the exact decimal
values of the end points (``Fraction(repr(x))``) and rounds each once.
"""
from fractions import Fraction

import numpy as np


def julia_linrange(a, b, n):
    """Float64 points of Julia's ``range(a, b, n)`` (grids.jl:206, 251-252, 310-312)."""
    n = int(n)
    if n < 1:
        raise ValueError("range length must be >= 1")
    if n == 1:
        return np.array([float(a)])
    fa = Fraction(repr(float(a)))
    fb = Fraction(repr(float(b)))
    step = (fb - fa) / (n - 1)
    return np.array([float(fa + i * step) for i in range(n)], dtype=np.float64)


def adapt_range(x, dtype):
    """Coordinates after ``adapt(backend{T}, ...)``: ``range(T(first(x)), T(last(x)), len)``
    (src/backends.jl:30).  For Float64 this reproduces the grid; for Float32 it is the
    correctly rounded Float32 linear range between the Float32 end points."""
    dtype = np.dtype(dtype)
    x = np.asarray(x, dtype=np.float64)
    if dtype == np.float64:
        return x.copy()
    n = len(x)
    a = Fraction(float(np.float32(x[0])))
    b = Fraction(float(np.float32(x[-1])))
    if n == 1:
        return np.array([np.float32(x[0])], dtype=np.float32)
    return np.array([np.float32(float(a + i * (b - a) / (n - 1))) for i in range(n)], dtype=np.float32)


class Grid:
    ndim = 0


class Grid1D(Grid):
    """1-D grid in z (grids.jl:182-210)."""
    ndim = 1

    def __init__(self, *, zmin, zmax, Nz):
        self.Nz = int(Nz)
        self.z = julia_linrange(zmin, zmax, Nz)
        self.dz = float(self.z[1] - self.z[0])
        self.Lz = float(self.z[-1] - self.z[0])
        self.Nx = self.Ny = 1
        self.dx = self.dy = 1.0

    @property
    def shape(self):
        return (self.Nz,)


class Grid2D(Grid):
    """2-D grid in the x-z plane, d/dy = 0 (grids.jl:216-258)."""
    ndim = 2

    def __init__(self, *, xmin, xmax, Nx, zmin, zmax, Nz):
        self.Nx, self.Nz = int(Nx), int(Nz)
        self.x = julia_linrange(xmin, xmax, Nx)
        self.z = julia_linrange(zmin, zmax, Nz)
        self.dx = float(self.x[1] - self.x[0])
        self.dz = float(self.z[1] - self.z[0])
        self.Lx = float(self.x[-1] - self.x[0])
        self.Lz = float(self.z[-1] - self.z[0])
        self.Ny = 1
        self.dy = 1.0

    @property
    def shape(self):
        return (self.Nx, self.Nz)


class Grid3D(Grid):
    """3-D grid (grids.jl:264-320)."""
    ndim = 3

    def __init__(self, *, xmin, xmax, Nx, ymin, ymax, Ny, zmin, zmax, Nz):
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.x = julia_linrange(xmin, xmax, Nx)
        self.y = julia_linrange(ymin, ymax, Ny)
        self.z = julia_linrange(zmin, zmax, Nz)
        self.dx = float(self.x[1] - self.x[0])
        self.dy = float(self.y[1] - self.y[0])
        self.dz = float(self.z[1] - self.z[0])
        self.Lx = float(self.x[-1] - self.x[0])
        self.Ly = float(self.y[-1] - self.y[0])
        self.Lz = float(self.z[-1] - self.z[0])

    @property
    def shape(self):
        return (self.Nx, self.Ny, self.Nz)


def make_grid(*, xmin=None, xmax=None, Nx=None, ymin=None, ymax=None, Ny=None, zmin, zmax, Nz):
    """``Grid(; ...)`` (grids.jl:145-176): 1-, 2- or 3-D depending on the keywords."""
    xargs = (xmin, xmax, Nx)
    yargs = (ymin, ymax, Ny)
    if all(v is None for v in xargs) and all(v is None for v in yargs):
        return Grid1D(zmin=zmin, zmax=zmax, Nz=Nz)
    if all(v is not None for v in xargs) and all(v is None for v in yargs):
        return Grid2D(xmin=xmin, xmax=xmax, Nx=Nx, zmin=zmin, zmax=zmax, Nz=Nz)
    if all(v is not None for v in xargs) and all(v is not None for v in yargs):
        return Grid3D(xmin=xmin, xmax=xmax, Nx=Nx, ymin=ymin, ymax=ymax, Ny=Ny,
                      zmin=zmin, zmax=zmax, Nz=Nz)
    raise ValueError(
        "Wrong set of arguments. To create a grid you need to define the following variables: "
        "1-D grid: zmin, zmax, Nz; 2-D grid: xmin, xmax, Nx, zmin, zmax, Nz; "
        "3-D grid: xmin, xmax, Nx, ymin, ymax, Ny, zmin, zmax, Nz"
    )
