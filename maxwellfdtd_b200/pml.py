"""CPML layer profiles (reference src/pml.jl)."""
import math
from dataclasses import dataclass

import numpy as np

from .constants import EPS0, MU0


@dataclass
class CPML:
    """``CPML(; thickness, kmax=1, alpha=10e-6, R0=10e-6, m=3)`` (pml.jl:1-40)."""
    thickness: float
    kmax: float = 1.0
    alpha: float = 10e-6
    R0: float = 10e-6
    m: int = 3


@dataclass
class PMLLayer:
    """``PMLLayer`` (pml.jl:46-52): ib is the 1-based boundary index, nb the point count.
    nb = 0 means no layer."""
    ib: int
    nb: int
    K: np.ndarray
    A: np.ndarray
    B: np.ndarray


def _params(L):
    if isinstance(L, CPML):
        return float(L.thickness), float(L.kmax), float(L.alpha), float(L.R0), int(L.m)
    return float(L), 1.0, 10e-6, 10e-6, 3


def _argmin_abs(x, v):
    return int(np.argmin(np.abs(x - v))) + 1   # 1-based, first minimum like Julia argmin


def _profile(x, idx, xb, Lx, dt, kmax, alpha, R0, m):
    eta0 = math.sqrt(MU0 / EPS0)
    smax = -(m + 1) * math.log(R0) / (2 * eta0 * Lx)
    n = len(idx)
    kappa = np.zeros(n)
    sigma = np.zeros(n)
    for j, i in enumerate(idx):
        r = (abs(x[i - 1] - xb) / Lx) ** m
        kappa[j] = 1 + (kmax - 1) * r
        sigma[j] = smax * r
    K = kappa
    B = np.exp(-(sigma / K + alpha) * dt / EPS0)
    A = sigma / (sigma * K + alpha * K ** 2) * (B - 1)
    return K, A, B


def left_layer(x, L, dt):
    """``LeftPMLLayer`` (pml.jl:57-90).  A zero thickness gives no layer (the reference
    leaves Nxb unassigned there; a layer with K=1, A=B=0 would change nothing)."""
    Lx, kmax, alpha, R0, m = _params(L)
    if Lx == 0:
        return PMLLayer(1, 0, np.ones(0), np.zeros(0), np.zeros(0))
    xb = x[0] + Lx
    ixb = _argmin_abs(x, xb)
    K, A, B = _profile(x, range(1, ixb + 1), xb, Lx, dt, kmax, alpha, R0, m)
    return PMLLayer(ixb, ixb, K, A, B)


def right_layer(x, L, dt):
    """``RightPMLLayer`` (pml.jl:93-127)."""
    Lx, kmax, alpha, R0, m = _params(L)
    n = len(x)
    if Lx == 0:
        return PMLLayer(n, 0, np.ones(0), np.zeros(0), np.zeros(0))
    xb = x[-1] - Lx
    ixb = _argmin_abs(x, xb)
    K, A, B = _profile(x, range(ixb, n + 1), xb, Lx, dt, kmax, alpha, R0, m)
    return PMLLayer(ixb, n - ixb + 1, K, A, B)


def _none_layer():
    return PMLLayer(1, 0, np.ones(0), np.zeros(0), np.zeros(0))


def make_pml(grid, pml, dt):
    """``PML(grid, pml, dt)`` (pml.jl:147-166, 194-221, 269-304).  Returns six layers in
    face order x-left, x-right, y-left, y-right, z-left, z-right."""
    single = not isinstance(pml, (tuple, list))
    layers = [_none_layer() for _ in range(6)]
    if grid.ndim == 1:
        Lz1, Lz2 = (pml, pml) if single else tuple(pml)
        layers[4] = left_layer(grid.z, Lz1, dt)
        layers[5] = right_layer(grid.z, Lz2, dt)
    elif grid.ndim == 2:
        Lx1, Lx2, Lz1, Lz2 = (pml,) * 4 if single else tuple(pml)
        layers[0] = left_layer(grid.x, Lx1, dt)
        layers[1] = right_layer(grid.x, Lx2, dt)
        layers[4] = left_layer(grid.z, Lz1, dt)
        layers[5] = right_layer(grid.z, Lz2, dt)
    else:
        Lx1, Lx2, Ly1, Ly2, Lz1, Lz2 = (pml,) * 6 if single else tuple(pml)
        layers[0] = left_layer(grid.x, Lx1, dt)
        layers[1] = right_layer(grid.x, Lx2, dt)
        layers[2] = left_layer(grid.y, Ly1, dt)
        layers[3] = right_layer(grid.y, Ly2, dt)
        layers[4] = left_layer(grid.z, Lz1, dt)
        layers[5] = right_layer(grid.z, Lz2, dt)
    return layers
