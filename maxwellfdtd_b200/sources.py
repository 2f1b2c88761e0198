"""Sources (reference src/sources.jl).

Waveforms are user functions of (coordinates..., t[, p]).  They cannot run on the device,
so they are tabulated on the host in double for every source point and step -- the value
the reference's add_source_kernel! computes at run time from the adapted (element type T)
coordinates and time (sources.jl:77-119, 190-232).  A SeparableWaveform(amplitude, pulse)
stores amplitude(coords) per point and pulse(t) per step instead of the full table.
"""
from dataclasses import dataclass
from typing import Any, Callable, Optional

import numpy as np

from . import _abi
from .constants import EPS0
from .geometry import cell_coords, geometry2indices

_COMP = {"Hx": 0, "Hy": 1, "Hz": 2, "Dx": 3, "Dy": 4, "Dz": 5, "Ex": 6, "Ey": 7, "Ez": 8}
COMPONENTS_3D = ("Hx", "Hy", "Hz", "Dx", "Dy", "Dz", "Ex", "Ey", "Ez")
COMPONENTS_2D = ("Hy", "Dx", "Dz", "Ex", "Ez")
COMPONENTS_2D_EY = ("Hx", "Hz", "Dy", "Ey")
COMPONENTS_1D = ("Hy", "Dx", "Ex")
POLARIZATIONS = ("Hy", "Ey")


def polarization_name(p):
    """The 2-D field set: "Hy" (Hy, Dx, Dz, Ex, Ez -- the reference's Field2D,
    fields.jl:36-55) or "Ey" (Hx, Hz, Dy, Ey; MFD_POL_EY in include/maxwellfdtd.h)."""
    p = str(p).lstrip(":")
    if p not in POLARIZATIONS:
        raise ValueError(f"polarization must be one of {POLARIZATIONS}, not {p!r}")
    return p


def field_components(ndim, polarization="Hy"):
    if ndim == 2 and polarization == "Ey":
        return COMPONENTS_2D_EY
    return {1: COMPONENTS_1D, 2: COMPONENTS_2D, 3: COMPONENTS_3D}[ndim]


def comp_index(name):
    name = str(name).lstrip(":")
    if name not in _COMP:
        raise ValueError(f"unknown field component {name!r}")
    return _COMP[name]


@dataclass
class SeparableWaveform:
    """waveform(coords..., t) = amplitude(coords...) * pulse(t)."""
    amplitude: Callable
    pulse: Callable


@dataclass
class SoftSource:
    """``SoftSource(; geometry, waveform, p=nothing, component, explicit=false)`` (sources.jl:9-37)."""
    geometry: Any
    waveform: Any
    component: str
    p: Any = None
    explicit: bool = False


@dataclass
class HardSource:
    """``HardSource(; geometry, waveform, p=nothing, component)`` (sources.jl:137-161)."""
    geometry: Any
    waveform: Any
    component: str
    p: Any = None


@dataclass
class TFSFSource:
    """``TFSFSource(fname)`` (sources.jl:250-266).  The incident data come from a record run
    (``solve(...; tfsf_record=True)``), stored as an .npz file with the reference's dataset
    names, or are given directly as that mapping (``data``)."""
    fname: Optional[str] = None
    data: Optional[dict] = None


@dataclass
class PointSourceStruct:
    """``SoftSourceStruct`` / ``HardSourceStruct`` (sources.jl:41-73, 165-186)."""
    kind: int            # 0 soft, 1 hard
    comp: int
    coeff: float
    cells: np.ndarray
    waveform: Any
    p: Any


def source_struct_point(source, grid, polarization="Hy"):
    cells = geometry2indices(source.geometry, grid)
    if len(cells) == 0:
        raise ValueError("I did not find any grid points which satisfy your source geometry.")
    comp = str(source.component).lstrip(":")
    if comp not in field_components(grid.ndim, polarization):
        raise ValueError(f"{grid.ndim}-D field has no component {comp}")
    if isinstance(source, SoftSource):
        if comp in ("Ex", "Ey", "Ez") and not source.explicit:
            comp = "D" + comp[1]
            coeff = EPS0
        else:
            coeff = 1.0
        return PointSourceStruct(0, comp_index(comp), coeff, cells, source.waveform, source.p)
    return PointSourceStruct(1, comp_index(comp), 1.0, cells, source.waveform, source.p)


def tabulate_waveform(src, grid, coords_T, t_T):
    """Waveform values in double for every point and step: returns (wave, amp, gt) with
    either wave [nt][npts] or the separable pair."""
    pts = cell_coords(grid, src.cells, coords_T)
    pts = tuple(np.asarray(c, dtype=np.float64) for c in pts)
    t = np.asarray(t_T, dtype=np.float64)
    wf = src.waveform
    if isinstance(wf, SeparableWaveform):
        amp = np.asarray(np.broadcast_to(wf.amplitude(*pts), pts[0].shape), dtype=np.float64)
        gt = np.asarray(np.broadcast_to(wf.pulse(t), t.shape), dtype=np.float64)
        return None, np.ascontiguousarray(amp), np.ascontiguousarray(gt)
    extra = () if src.p is None else (src.p,)
    try:
        with np.errstate(all="ignore"):
            wave = wf(*[c[None, :] for c in pts], t[:, None], *extra)
        wave = np.broadcast_to(np.asarray(wave, dtype=np.float64), (len(t), len(src.cells)))
    except (TypeError, ValueError):
        wave = np.empty((len(t), len(src.cells)))
        for it in range(len(t)):
            for j in range(len(src.cells)):
                wave[it, j] = wf(*[float(c[j]) for c in pts], float(t[it]), *extra)
    return np.ascontiguousarray(wave, dtype=np.float64), None, None


# ----------------------------------------------------------------------------------------
# TFSF
# ----------------------------------------------------------------------------------------
TFSF_NAMES_1D = ("incHy_1", "incEx_1", "incHy_2", "incEx_2")
TFSF_NAMES_2D = ("incHy_1z", "incEz_1z", "incHy_2z", "incEz_2z",
                 "incHy_x1", "incEx_x1", "incHy_x2", "incEx_x2")
TFSF_NAMES_3D = ("incHy_1yz", "incHz_1yz", "incEy_1yz", "incEz_1yz",
                 "incHy_2yz", "incHz_2yz", "incEy_2yz", "incEz_2yz",
                 "incHx_x1z", "incHz_x1z", "incEx_x1z", "incEz_x1z",
                 "incHx_x2z", "incHz_x2z", "incEx_x2z", "incEz_x2z",
                 "incHx_xy1", "incHy_xy1", "incEx_xy1", "incEy_xy1",
                 "incHx_xy2", "incHy_xy2", "incEx_xy2", "incEy_xy2")


# The second 2-D field set: Hz, Ey on the x faces and Hx, Ey on the z faces, over the nodes
# i1..i2 (the 3-D faces 1yz, 2yz, xy1, xy2 restricted to those components).
TFSF_NAMES_2D_EY = ("incHz_1z", "incEy_1z", "incHz_2z", "incEy_2z",
                    "incHx_x1", "incEy_x1", "incHx_x2", "incEy_x2")


def tfsf_names(ndim, polarization="Hy"):
    if ndim == 2 and polarization == "Ey":
        return TFSF_NAMES_2D_EY
    return {1: TFSF_NAMES_1D, 2: TFSF_NAMES_2D, 3: TFSF_NAMES_3D}[ndim]


def _argmin1(x, v):
    return int(np.argmin(np.abs(np.asarray(x) - v))) + 1


def box_indices(grid, box, coords=None):
    """1-based box indices from box coordinates (sources.jl:298-300, 428-432, 629-635)."""
    cs = coords
    if grid.ndim == 1:
        z = grid.z if cs is None else cs[0]
        z1, z2 = box
        return (1, 1, _argmin1(z, z1)), (1, 1, _argmin1(z, z2))
    if grid.ndim == 2:
        x = grid.x if cs is None else cs[0]
        z = grid.z if cs is None else cs[1]
        x1, x2, z1, z2 = box
        return (_argmin1(x, x1), 1, _argmin1(z, z1)), (_argmin1(x, x2), 1, _argmin1(z, z2))
    x = grid.x if cs is None else cs[0]
    y = grid.y if cs is None else cs[1]
    z = grid.z if cs is None else cs[2]
    x1, x2, y1, y2, z1, z2 = box
    return ((_argmin1(x, x1), _argmin1(y, y1), _argmin1(z, z1)),
            (_argmin1(x, x2), _argmin1(y, y2), _argmin1(z, z2)))


def _interp_axis(knots, values, q, axis):
    """Linear interpolation of ``values`` along ``axis`` at points q with constant (Flat)
    extrapolation -- Interpolations.jl ``linear_interpolation(...; extrapolation_bc=Flat())``
    on one axis of a gridded table."""
    knots = np.asarray(knots, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    n = len(knots)
    if values.shape[axis] == 1:
        return np.asarray(values)    # constant along this axis (one knot, or given broadcast)
    if n == len(q) and np.array_equal(knots, q):
        return np.asarray(values)    # queries on the knots: interpolation is the identity
    qc = np.clip(q, knots[0], knots[-1])
    i = np.clip(np.searchsorted(knots, qc, side="right") - 1, 0, n - 2)
    w = (qc - knots[i]) / (knots[i + 1] - knots[i])
    a = np.take(values, i, axis=axis)
    b = np.take(values, i + 1, axis=axis)
    shape = [1] * values.ndim
    shape[axis] = len(q)
    w = w.reshape(shape)
    return a * (1 - w) + b * w


def _interp_grid(knot_list, values, query_list):
    out = np.asarray(values, dtype=np.float64)
    for ax, (k, q) in enumerate(zip(knot_list, query_list)):
        out = _interp_axis(k, out, q, ax)
    return out


def load_tfsf_data(source):
    if source.data is not None:
        return {k: np.asarray(v) for k, v in source.data.items()}
    with np.load(source.fname) as f:
        return {k: f[k] for k in f.files}


def _compact(r, extent):
    """r: resampled incident data (a, b, nt) of a face of `extent` (a, b), an axis of extent 1
    meaning constant along it.  Axes whose values are the same everywhere are dropped too;
    returns the C-ordered values per step [nt][...] and the MFD_INC_* layout
    (include/maxwellfdtd.h)."""
    if r.shape[0] > 1 and np.array_equal(r, np.broadcast_to(r[:1], r.shape)):
        r = r[:1]
    if r.shape[1] > 1 and np.array_equal(r, np.broadcast_to(r[:, :1], r.shape)):
        r = r[:, :1]
    A, B, nt = r.shape
    shape = (_abi.MFD_INC_UNIFORM if A == 1 and B == 1 else _abi.MFD_INC_ALONG_B if A == 1
             else _abi.MFD_INC_ALONG_A if B == 1 else _abi.MFD_INC_FULL)
    return np.ascontiguousarray(np.transpose(r, (2, 1, 0)).reshape(nt, -1)), shape


def tfsf_struct(source, grid, t, polarization="Hy"):
    """``SourceStruct(::TFSFSource, ...)`` (sources.jl:284-317, 408-466, 592-710): box
    indices on this grid and incident data resampled onto (face coordinates, t), dense in t.
    Arrays are returned C-ordered [nt][face extent] (the reference's (a, b, Nt) column-major),
    each in its compact layout when its values do not vary along a face axis (the dataset may
    give such an axis with extent 1); returns (i1, i2, arrays, layouts)."""
    d = load_tfsf_data(source)
    box = tuple(float(v) for v in np.asarray(d["box"]).ravel())
    tex = np.asarray(d["t"], dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    i1, i2 = box_indices(grid, box)
    arrays = []
    shapes = []
    if grid.ndim == 1:
        for name in TFSF_NAMES_1D:
            v = np.asarray(d[name], dtype=np.float64).ravel()
            arrays.append(_interp_axis(tex, v, t, 0).reshape(len(t), 1))
            shapes.append(_abi.MFD_INC_FULL)
        return i1, i2, arrays, shapes
    if grid.ndim == 2:
        xex = np.asarray(d["x"], dtype=np.float64)
        zex = np.asarray(d["z"], dtype=np.float64)
        ix1, iz1 = i1[0], i1[2]
        ix2, iz2 = i2[0], i2[2]
        names = tfsf_names(2, polarization)
        if any(n not in d for n in names):
            raise ValueError(f"the TFSF data do not hold the {polarization} polarisation's arrays "
                             + ", ".join(names))
        e = 1 if polarization == "Ey" else 0   # node ranges i1..i2 in the Ey field set
        zq = grid.z[iz1 - 1:iz2 - 1 + e]
        xq = grid.x[ix1 - 1:ix2 - 1 + e]
        for name in names:
            v = np.asarray(d[name], dtype=np.float64)   # (face, Nt) column-major in the file
            v = _as_col_major(v, 2)
            knots, q = (zex, zq) if name.endswith("z") else (xex, xq)
            r = _interp_grid([knots, tex], v, [q, t])      # (face, nt)
            arr, sh = _compact(r[:, None, :], (len(q), 1))
            arrays.append(arr)
            shapes.append(sh)
        return i1, i2, arrays, shapes
    xex = np.asarray(d["x"], dtype=np.float64)
    yex = np.asarray(d["y"], dtype=np.float64)
    zex = np.asarray(d["z"], dtype=np.float64)
    (ix1, iy1, iz1), (ix2, iy2, iz2) = i1, i2
    X, Y, Z = grid.x, grid.y, grid.z
    xf, xh = X[ix1 - 1:ix2], X[ix1 - 1:ix2 - 1]
    yf, yh = Y[iy1 - 1:iy2], Y[iy1 - 1:iy2 - 1]
    zf, zh = Z[iz1 - 1:iz2], Z[iz1 - 1:iz2 - 1]
    # (knots a, knots b, query a, query b) per array, sources.jl:642-699
    spec = []
    for _ in range(2):   # 1yz, 2yz
        spec += [(yex, zex[:-1], yf, zh), (yex[:-1], zex, yh, zf), (yex[:-1], zex, yh, zf), (yex, zex[:-1], yf, zh)]
    for _ in range(2):   # x1z, x2z
        spec += [(xex, zex[:-1], xf, zh), (xex[:-1], zex, xh, zf), (xex[:-1], zex, xh, zf), (xex, zex[:-1], xf, zh)]
    for _ in range(2):   # xy1, xy2
        spec += [(xex, yex[:-1], xf, yh), (xex[:-1], yex, xh, yf), (xex[:-1], yex, xh, yf), (xex, yex[:-1], xf, yh)]
    for name, (ka, kb, qa, qb) in zip(TFSF_NAMES_3D, spec):
        v = _as_col_major(np.asarray(d[name], dtype=np.float64), 3)
        r = _interp_grid([ka, kb, tex], v, [qa, qb, t])    # (a, b, nt)
        arr, sh = _compact(r, (len(qa), len(qb)))
        arrays.append(arr)
        shapes.append(sh)
    return i1, i2, arrays, shapes


def _as_col_major(v, nd):
    """Arrays saved by this package's record path are C-ordered [nt][b][a]; reorder to the
    reference's (a, b, nt) view."""
    if v.ndim == nd:
        return np.transpose(v, tuple(range(nd - 1, -1, -1)))
    raise ValueError("TFSF dataset has the wrong number of dimensions")
