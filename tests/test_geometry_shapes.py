"""Analytic shapes evaluated by the library (mfd_shape, csrc/geometry.cuh) instead of the
host: the same map as the host evaluation of the same expression, bit for bit, including
cells exactly on a shape's boundary; later shapes overwrite earlier ones (models.jl:91-98);
whole solves with shapes equal solves with the host map."""
import numpy as np
import pytest

import cases as C
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import _abi


def _grid(ndim, n=(24, 20, 18), d=25e-9):
    if ndim == 3:
        return C.grid3(n, d)
    if ndim == 2:
        return C.grid2((n[0], n[2]), d)
    return C.grid1(n[2], d)


def _shape_models(ndim):
    """Materials on shapes whose boundaries pass through grid points (r = 4 cells from a
    grid point), in an order where later ones overlap earlier ones."""
    g = _grid(ndim)
    d = 25e-9
    pt = lambda *v: tuple(v[:ndim]) if ndim == 3 else ((v[0], v[2]) if ndim == 2 else (v[2],))
    ball = M.Ball(pt(g.x[12] if ndim > 1 else 0, g.y[10] if ndim == 3 else 0, g.z[9]), 4 * d)
    box = M.Box(pt(-3 * d, -2 * d, -1.5 * d), pt(2.5 * d, 3 * d, 0.0))
    ell = M.Ellipsoid(pt(0.0, 0.0, 2 * d), pt(5 * d, 3 * d, 2 * d))
    half = M.HalfSpace(pt(0.0, 0.0, 1.0), 5 * d)
    shapes = [ball, box, ell, half]
    if ndim == 3:
        shapes.append(M.Cylinder((g.x[4], g.y[5]), 3 * d, -4 * d, 6 * d))
    mats = [M.Material(geometry=s, eps=1.5 + 0.5 * k) for k, s in enumerate(shapes)]
    mats[1] = M.Material(geometry=box, eps=3.0, chi=M.DebyeSusceptibility(deps=1.0, tau=1e-14))
    src = M.SoftSource(geometry=C._geo_point(ndim, (0.0, 0.0, -100e-9)), waveform=C._src_wave(ndim), component="Ex")
    dt = 0.5 / C.C0 / np.sqrt(ndim / d ** 2)
    return M.Model(g, src, tmax=(30 - 0.5) * dt, pml=100e-9, material=mats)


@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_shapes_on_host_and_in_oracle(ndim, oracle_lib):
    model = _shape_models(ndim)
    assert model.shapes() is not None
    host = model.geometry.ravel(order="F")
    assert len(np.unique(host)) >= 4                 # every shape is present, overlaps resolved
    b, _ = model.build_desc(np.float64, None)
    assert b.desc.nshape > 0 and not b.desc.geometry
    st = _abi.Stepper(oracle_lib, b, np.float64)
    assert np.array_equal(st.read_geometry(), host)
    st.close()
    got = C.run_all(model, oracle_lib, np.float64)
    b2, _ = model.build_desc(np.float64, None, device_geometry=False)
    assert b2.desc.nshape == 0
    model._geometry = None
    ref = C.run_all(_HostMap(model), oracle_lib, np.float64)
    for k in ref:
        assert np.array_equal(ref[k], got[k]), k


class _HostMap:
    """A model passed with its host map (the shapes hidden)."""

    def __init__(self, model):
        self.__dict__.update(model.__dict__)
        self._m = model

    def __getattr__(self, k):
        return getattr(self._m, k)

    def build_desc(self, *a, **kw):
        kw["device_geometry"] = False
        return self._m.build_desc(*a, **kw)


def test_shape_boundaries_exact():
    """A cell exactly at distance r is inside; the expression is the header's."""
    g = _grid(3)
    d = 25e-9
    ball = M.Ball((g.x[10], g.y[10], g.z[9]), 4 * d)
    m = ball(g.x[:, None, None], g.y[None, :, None], g.z[None, None, :])
    a = g.x[14] - g.x[10]
    assert m[14, 10, 9] == bool(a * a + 0.0 + 0.0 <= (4 * d) * (4 * d))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_device_map_equals_host(ndim, dtype, oracle_lib, gpu_lib):
    model = _shape_models(ndim)
    b, _ = model.build_desc(dtype, None)
    st = _abi.Stepper(gpu_lib, b, dtype)
    dev = st.read_geometry()
    st.close()
    assert np.array_equal(dev, model.geometry.ravel(order="F"))
    got = C.run_all(model, gpu_lib, dtype)
    ref = C.run_all(_HostMap(model), oracle_lib, dtype)
    for k in ref:
        assert np.array_equal(ref[k], got[k]), k


@pytest.mark.gpu
def test_device_geometry_large_grid(gpu_lib):
    """The 256^3 plasmonics sphere as a Ball: the device map equals the host map."""
    n, dx = 256, 2e-9
    L = (n - 1) * dx / 2
    g = M.Grid(xmin=-L, xmax=L, Nx=n, ymin=-L, ymax=L, Ny=n, zmin=-L, zmax=L, Nz=n)
    mat = M.Material(geometry=M.Ball((0.0, 0.0, 0.0), 60e-9), eps=9.0,
                     chi=[M.DrudeSusceptibility(wp=1.37e16, gamma=1.07e14)])
    src = M.SoftSource(geometry=(0.0, 0.0, -100e-9), waveform=lambda x, y, z, t: np.sin(1e15 * t), component="Ex")
    model = M.Model(g, src, tmax=3 * 0.5 / M.C0 / np.sqrt(3 / dx ** 2), pml=12 * dx, material=mat)
    b, _ = model.build_desc(np.float32, None)
    st = _abi.Stepper(gpu_lib, b, np.float32)
    dev = st.read_geometry()
    st.run(1, model.Nt)
    st.close()
    assert np.array_equal(dev, model.geometry.ravel(order="F")) and dev.sum() > 0
