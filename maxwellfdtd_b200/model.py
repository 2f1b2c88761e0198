"""Model setup and the run loop (reference src/models.jl:1-242, src/outputs.jl).

``Model(grid, source; tmax, CN, bc, pml, material)`` computes, on the host and in Float64,
everything the reference computes there: the time step, the time grid, source points,
CPML profiles, the material map and the material coefficients.  ``solve`` hands the
result to the CUDA library through the C ABI (include/maxwellfdtd.h) and runs the time
loop on the device.
"""
import math
import os
from dataclasses import dataclass

import numpy as np

from . import _abi
from .constants import C0
from .geometry import Shape, geometry2bool
from .grids import adapt_range
from .materials import IonizationRate, Material, PowerLawRate, material_struct
from .monitors import FieldMonitor, SpectralMonitor, monitor_struct
from .pml import make_pml
from .sources import (HardSource, SoftSource, TFSFSource, box_indices, comp_index, field_components,
                      polarization_name, source_struct_point, tabulate_waveform, tfsf_names, tfsf_struct)

_BC = {"periodic": 1, "dirichlet": 2, "neumann": 3}


def bc2int(bc):
    """``bc2int`` (models.jl:1199-1212)."""
    key = str(bc).lstrip(":")
    if key not in _BC:
        raise ValueError("Wrong 'bc' value. It can be either ':periodic', ':dirichlet', or ':neumann'.")
    return _BC[key]


def time_step(grid, CN):
    """``time_step`` (models.jl:1181-1196)."""
    if grid.ndim == 1:
        return CN / C0 / math.sqrt(1 / (grid.dz * grid.dz))
    if grid.ndim == 2:
        return CN / C0 / math.sqrt(1 / (grid.dx * grid.dx) + 1 / (grid.dz * grid.dz))
    return CN / C0 / math.sqrt(1 / (grid.dx * grid.dx) + 1 / (grid.dy * grid.dy) + 1 / (grid.dz * grid.dz))


def time_range(dt, tmax):
    """Julia ``range(start=0, step=dt, stop=tmax)`` for a step with no exact small rational
    form: length round(tmax/dt)+1, minus one if that overshoots tmax; t[i] = (i-1)*dt."""
    lf = tmax / dt
    if lf < 0:
        n = 0
    elif lf == 0:
        n = 1
    else:
        n = int(round(lf)) + 1
        stop_ = (n - 1) * dt
        if 0 < tmax < stop_:
            n -= 1
    return np.arange(n, dtype=np.float64) * dt


def adapt_time(t, dtype):
    """Time range after adapt(backend{T}): ``range(T(first(t)), T(last(t)), len)``."""
    from fractions import Fraction
    dtype = np.dtype(dtype)
    n = len(t)
    if n < 2:
        return np.asarray(t, dtype=dtype)
    last = Fraction(float(dtype.type(t[-1])))
    return np.array([float(last * i / (n - 1)) for i in range(n)], dtype=np.float64).astype(dtype)


class Model:
    """``Model(grid, source; tmax, CN=0.5, bc=:periodic, pml=0, material=nothing)``.
    ``polarization`` chooses the field set of a 2-D model: "Hy" (Hy, Dx, Dz, Ex, Ez, the
    reference's) or "Ey" (Hx, Hz, Dy, Ey, which the reference does not have)."""

    def __init__(self, grid, source, *, tmax, CN=0.5, bc="periodic", pml=0, material=None, polarization="Hy"):
        self.grid = grid
        self.polarization = polarization_name(polarization)
        if grid.ndim != 2 and self.polarization != "Hy":
            raise ValueError("polarization applies to 2-D models")
        self.dt = time_step(grid, CN)
        self.t = time_range(self.dt, tmax)
        self.Nt = len(self.t)
        if self.Nt < 1:
            raise ValueError("tmax gives no time steps")
        srcs = list(source) if isinstance(source, (list, tuple)) else [source]
        self.point_sources = []
        self.tfsf = None
        self.tfsf_order = 0
        for s in srcs:
            if isinstance(s, TFSFSource):
                if self.tfsf is not None:
                    raise ValueError("one TFSF source per model")
                self.tfsf = tfsf_struct(s, grid, self.t, self.polarization)
                self.tfsf_order = len(self.point_sources)
            elif isinstance(s, (SoftSource, HardSource)):
                self.point_sources.append(source_struct_point(s, grid, self.polarization))
            else:
                raise TypeError(f"unknown source type {type(s).__name__}")
        nfaces = 2 * grid.ndim
        if isinstance(bc, (list, tuple)):
            if len(bc) != nfaces:
                raise ValueError(f"bc needs {nfaces} values for a {grid.ndim}-D grid")
            codes = [bc2int(b) for b in bc]
        else:
            codes = [bc2int(bc)] * nfaces
        faces = {1: [4, 5], 2: [0, 1, 4, 5], 3: [0, 1, 2, 3, 4, 5]}[grid.ndim]
        self.bcs = [1] * 6
        for f, c in zip(faces, codes):
            self.bcs[f] = c
        self.pml = make_pml(grid, pml, self.dt)
        mats = [] if material is None else (list(material) if isinstance(material, (list, tuple)) else [material])
        if len(mats) > 255:
            raise ValueError("at most 255 materials")
        self._mat_geometries = [m.geometry for m in mats]
        self._geometry = None
        self.materials = [material_struct(m, self.dt) for m in mats]
        self.Mh, self.Me, self.Md1, self.Md2 = self.dt / 1.25663706212e-6, 1 / 8.8541878128e-12, 1.0, self.dt
        self.isplasma = any(m.isplasma for m in self.materials)

    @property
    def geometry(self):
        """The material index map (models.jl:85-98: later materials win), evaluated on the
        host when first asked for.  A model whose materials are all analytic shapes
        (geometry.Shape) does not need it: its descriptor passes the shapes and the library
        builds the map on the device."""
        if self._geometry is None:
            geom = np.zeros(self.grid.shape, dtype=np.uint8)
            for imat, g in enumerate(self._mat_geometries, start=1):
                geom[geometry2bool(g, self.grid)] = imat
            self._geometry = geom
        return self._geometry

    def shapes(self):
        """[(material index, Shape)] when every material's geometry is a Shape, else None."""
        if self._mat_geometries and all(isinstance(g, Shape) for g in self._mat_geometries):
            return [(i, g) for i, g in enumerate(self._mat_geometries, start=1)]
        return None

    # ------------------------------------------------------------------------------------
    def coords(self, dtype):
        g = self.grid
        if g.ndim == 1:
            return (adapt_range(g.z, dtype),)
        if g.ndim == 2:
            return (adapt_range(g.x, dtype), adapt_range(g.z, dtype))
        return (adapt_range(g.x, dtype), adapt_range(g.y, dtype), adapt_range(g.z, dtype))

    def build_desc(self, dtype, monitors=(), tfsf_box=None, rho_fp64=True, device=0, host_alloc=None, mode="exact",
                   device_geometry=None):
        """C descriptor for this model in element type ``dtype`` plus host-side metadata.
        ``host_alloc(n, dtype)`` provides the storage of the large input arrays (e.g.
        page-locked memory).  ``mode`` is the arithmetic of the field updates: "exact" (the
        reference's operation order, bit for bit) or "fast" (the tolerance mode,
        MFD_MODE_FAST in include/maxwellfdtd.h).  ``device_geometry``: None passes the
        materials' shapes for the device to evaluate when every geometry is a Shape (else
        the host map), True requires that, False always passes the host map."""
        if mode not in ("exact", "fast"):
            raise ValueError("mode must be 'exact' or 'fast'")
        dtype = np.dtype(dtype)
        g = self.grid
        b = _abi.DescBuilder(host_alloc)
        d = b.desc
        d.abi_version = _abi.ABI_VERSION
        d.ndim = g.ndim
        d.dtype = _abi.MFD_F64 if dtype == np.float64 else _abi.MFD_F32
        d.nx, d.ny, d.nz = g.Nx, g.Ny, g.Nz
        d.dx, d.dy, d.dz = g.dx, g.dy, g.dz
        d.dt = self.dt
        d.nt = self.Nt
        for f in range(6):
            d.bc[f] = self.bcs[f]
            L = self.pml[f]
            d.pml[f].ib = L.ib
            d.pml[f].nb = L.nb
            if L.nb:
                d.pml[f].K = _abi.dptr(b.arr(L.K, np.float64))
                d.pml[f].A = _abi.dptr(b.arr(L.A, np.float64))
                d.pml[f].B = _abi.dptr(b.arr(L.B, np.float64))
        d.Mh0, d.Me0, d.Md10, d.Md20 = self.Mh, self.Me, self.Md1, self.Md2
        shapes = self.shapes() if device_geometry is not False else None
        if device_geometry and shapes is None:
            raise ValueError("device_geometry needs every material's geometry to be a Shape")
        if shapes:   # the library builds the map on the device
            sarr = (_abi.Shape * len(shapes))()
            b.keep.append(sarr)
            for k, (imat, shp) in enumerate(shapes):
                sarr[k].kind = shp.kind
                sarr[k].material = imat
                for j, v in enumerate(shp.params(g.ndim)):
                    sarr[k].p[j] = v
            d.nshape = len(shapes)
            d.shapes = sarr
            axes = (g.x, g.y, g.z) if g.ndim == 3 else (g.x, None, g.z) if g.ndim == 2 else (None, None, g.z)
            for k, c in enumerate(axes):
                if c is not None:
                    d.coords[k] = _abi.dptr(b.arr(np.asarray(c, dtype=np.float64), np.float64))
        else:
            geo = b.arr(self.geometry.ravel(order="F"), np.uint8)
            d.geometry = geo.ctypes.data_as(_abi.C.POINTER(_abi.C.c_uint8))
        nm = len(self.materials)
        d.nmat = nm
        if nm:
            arr = (_abi.Material * nm)()
            b.keep.append(arr)
            for i, m in enumerate(self.materials):
                a = arr[i]
                a.Mh, a.Me, a.Md1, a.Md2 = m.Mh, m.Me, m.Md1, m.Md2
                a.nq = m.nq
                if m.nq:
                    a.Aq = _abi.dptr(b.arr(m.Aq, np.float64))
                    a.Bq = _abi.dptr(b.arr(m.Bq, np.float64))
                    a.Cq = _abi.dptr(b.arr(m.Cq, np.float64))
                a.kerr, a.Mk2, a.Mk3 = int(m.iskerr), m.Mk2, m.Mk3
                a.plasma = int(m.isplasma)
                if m.isplasma:
                    a.Rava, a.ksi, a.rho0, a.Ap, a.Bp, a.Cp, a.Ma = m.Rava, m.ksi, m.rho0, m.Ap, m.Bp, m.Cp, m.Ma
                    if isinstance(m.rate, PowerLawRate):
                        a.rate_kind = _abi.MFD_RATE_POWER
                        a.rate_order, a.rate_log10c = float(m.rate.order), float(m.rate.log10c)
                    else:
                        a.rate_kind = _abi.MFD_RATE_TABLE
                        a.rate_n = len(m.rate.x)
                        a.rate_x = _abi.dptr(b.arr(m.rate.x, np.float64))
                        a.rate_y = _abi.dptr(b.arr(m.rate.y, np.float64))
            d.mats = arr
        d.rho_fp64 = int(bool(rho_fp64))
        coords_T = self.coords(dtype)
        t_T = adapt_time(self.t, dtype)
        ns = len(self.point_sources)
        d.nsrc = ns
        if ns:
            sarr = (_abi.Source * ns)()
            b.keep.append(sarr)
            for i, s in enumerate(self.point_sources):
                wave, amp, gt = tabulate_waveform(s, g, coords_T, t_T)
                e = sarr[i]
                e.kind, e.comp, e.coeff = s.kind, s.comp, s.coeff
                e.npts = len(s.cells)
                e.cells = b.arr(s.cells, np.int64).ctypes.data_as(_abi.C.POINTER(_abi.C.c_int64))
                if wave is not None:
                    e.wave = _abi.dptr(b.arr(wave, np.float64))
                else:
                    e.amp = _abi.dptr(b.arr(amp, np.float64))
                    e.gt = _abi.dptr(b.arr(gt, np.float64))
            d.srcs = sarr
        if self.tfsf is not None:
            i1, i2, arrays, shapes = self.tfsf
            d.tfsf.enabled = 1
            d.tfsf.order = self.tfsf_order
            for a in range(3):
                d.tfsf.i1[a], d.tfsf.i2[a] = i1[a], i2[a]
            for k, (v, sh) in enumerate(zip(arrays, shapes)):
                d.tfsf.inc[k] = b.arr(v, dtype).ctypes.data
                d.tfsf.shape[k] = sh
        mon_meta = []
        monitors = [] if monitors is None else (list(monitors) if isinstance(monitors, (list, tuple)) else [monitors])
        if monitors:
            marr = (_abi.Monitor * len(monitors))()
            b.keep.append(marr)
            for i, mon in enumerate(monitors):
                ms = monitor_struct(mon, g, coords_T, t_T, dtype)
                e = marr[i]
                e.kind, e.sum = ms["kind"], int(ms["sum"])
                e.npts = len(ms["cells"])
                e.cells = b.arr(ms["cells"], np.int64).ctypes.data_as(_abi.C.POINTER(_abi.C.c_int64))
                if ms["kind"] == 1:
                    e.nw = ms["dft"].Nw
                    e.phasor = _abi.dptr(b.arr(ms["dft"].phasor, np.float64))
                mon_meta.append(ms)
            d.nmon = len(monitors)
            d.mons = marr
        rec = None
        if tfsf_box is not None:
            i1, i2 = box_indices(g, tfsf_box, coords_T)
            d.tfsf_record = 1
            for a in range(3):
                d.rec_i1[a], d.rec_i2[a] = i1[a], i2[a]
            rec = (tuple(float(v) for v in tfsf_box), i1, i2)
        d.device = device
        d.mode = _abi.MFD_MODE_FAST if mode == "fast" else _abi.MFD_MODE_EXACT
        d.polarization = _abi.MFD_POL_EY if self.polarization == "Ey" else _abi.MFD_POL_HY
        meta = {"coords_T": coords_T, "t_T": t_T, "monitors": mon_meta, "record": rec}
        return b, meta


# ----------------------------------------------------------------------------------------
# Backends
# ----------------------------------------------------------------------------------------
_LIB_CACHE = {}


def library_path():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmaxwellfdtd_b200.so")


def load_library(path=None):
    """The CUDA library (fails loudly when it has not been built: there is no CPU path).
    MFD_LIBRARY names another build of the same library."""
    path = path or os.environ.get("MFD_LIBRARY") or library_path()
    if path not in _LIB_CACHE:
        if not os.path.exists(path):
            raise RuntimeError(f"CUDA library {path} is not built; run __graft_entry__.build()")
        _LIB_CACHE[path] = _abi.Library(path, "mfd_")
    return _LIB_CACHE[path]


class B200:
    """Backend running the time-step path on a B200 GPU: ``B200(np.float32)`` or
    ``B200(np.float64)``; ``B200()`` is single precision like the reference's ``GPU()``
    (src/backends.jl:19-23).  ``library`` lets a caller supply another library object that
    exports the same C API.  ``mode="fast"`` selects the tolerance-mode field updates
    (reciprocal multiplies and fused multiply-adds, within relative L2 1e-5 in float32 and
    1e-12 in float64 of the exact order); the default "exact" keeps the reference's operation
    order bit for bit."""

    def __init__(self, dtype=np.float32, device=0, rho_fp64=True, library=None, mode="exact"):
        self.dtype = np.dtype(dtype)
        if self.dtype not in (np.dtype(np.float32), np.dtype(np.float64)):
            raise ValueError("B200 backend supports float32 and float64")
        if mode not in ("exact", "fast"):
            raise ValueError("mode must be 'exact' or 'fast'")
        self.device = device
        self.rho_fp64 = rho_fp64
        self.mode = mode
        self._library = library

    def library(self):
        return self._library if self._library is not None else load_library()


# ----------------------------------------------------------------------------------------
# solve
# ----------------------------------------------------------------------------------------
def output_times(t, nstride, nframes, dtout):
    """``output_times`` (outputs.jl:491-518): indices (1-based) of the snapshot steps."""
    Nt = len(t)
    given = [v is not None for v in (nstride, nframes, dtout)]
    if sum(given) == 0:
        raise ValueError("One of 'nstride', 'nframes', or 'dtout' should be specified.")
    if sum(given) > 1:
        raise ValueError("Only one of 'nstride', 'nframes', or 'dtout' can be specified.")
    if nstride is not None:
        if nstride >= Nt:
            nstride = Nt - 1
    elif nframes is not None:
        nstride = 1 if nframes >= Nt else int(round(Nt / nframes))
    else:
        tmax = float(t[-1])
        nstride = 1 if dtout >= tmax else int(round(Nt / (tmax / dtout)))
    nstride = max(int(nstride), 1)
    return list(range(1, Nt + 1, nstride))


class Field:
    """Field components of a solved model as grid-shaped arrays (Fortran order)."""

    def __init__(self, arrays):
        self.__dict__.update(arrays)

    def __getitem__(self, k):
        return self.__dict__[k]


@dataclass
class Solution:
    model: Model
    field: Field
    out: dict
    t: np.ndarray
    dtype: np.dtype


def _grid_shape(grid):
    return grid.shape


def solve(model, *, backend=None, fname=None, nframes=None, nstride=None, dtout=None,
          components=None, monitors=None, tfsf_record=False, tfsf_fname=None, tfsf_box=None,
          max_chunk=4096):
    """``solve!(model; backend, ...)`` (models.jl:166-242).  Returns a Solution whose
    ``field`` holds the final fields and whose ``out`` holds what the reference writes to
    its output file (Sa, E2, rho_end, JE, field snapshots, monitors); with ``fname`` the
    same datasets are saved: an HDF5 file in the reference's layout when the name ends in
    .hdf, .h5 or .hdf5 (the reference's default is "out.hdf"), else an .npz file."""
    backend = backend or B200()
    dtype = backend.dtype
    g = model.grid
    if tfsf_record and tfsf_box is None:
        raise ValueError("tfsf_record needs tfsf_box")
    builder, meta = model.build_desc(dtype, monitors, tfsf_box if tfsf_record else None,
                                     rho_fp64=backend.rho_fp64, device=getattr(backend, "device", 0),
                                     mode=getattr(backend, "mode", "exact"))
    st = _abi.Stepper(backend.library(), builder, dtype)
    try:
        return _run(model, st, meta, dtype, fname, nframes, nstride, dtout, components, monitors,
                    tfsf_record, tfsf_fname, max_chunk)
    finally:
        st.close()


def _run(model, st, meta, dtype, fname, nframes, nstride, dtout, components, monitors,
         tfsf_record, tfsf_fname, max_chunk):
    g = model.grid
    shape = _grid_shape(g)
    Nt = model.Nt
    t_T = meta["t_T"]
    comps_all = [c for c in field_components(g.ndim, model.polarization) if not c.startswith("D")]
    isfields = not (nstride is None and nframes is None and dtout is None)
    out_steps = output_times(t_T, nstride, nframes, dtout) if isfields else []
    if components is None:
        components = comps_all
    else:
        components = [str(c).lstrip(":") for c in components]
        for c in components:
            if c not in comps_all:
                raise ValueError(f"You asked to output {c} field component, but {g.ndim}-D field has only "
                                 + ", ".join(":" + x for x in comps_all) + " components.")
    isgeometry = bool(np.any(model.geometry > 0))
    out = {"t": np.asarray(t_T), "pml": np.array([model.pml[f].ib for f in
                                                   {1: [4, 5], 2: [0, 1, 4, 5], 3: range(6)}[g.ndim]])}
    for name, c in zip({1: ["z"], 2: ["x", "z"], 3: ["x", "y", "z"]}[g.ndim], meta["coords_T"]):
        out[name] = np.asarray(c)
    if isgeometry:
        out["geometry"] = model.geometry.astype(np.int64)
    snaps = {c: [] for c in components}
    if isfields and model.isplasma:
        snaps["rho"] = []
    # frames on a copy stream while the run goes on, when the library takes snapshots (rho
    # of plasma models is read at the output steps)
    device_frames = isfields and getattr(st.lib, "has_snapshots", False) and "rho" not in snaps
    if device_frames:
        # an ordinary host array: page-locking one for a single solve costs more than the
        # faster copies save (a caller of mfd_set_snapshots that reuses page-locked memory
        # gets the frames fully hidden behind the steps)
        buf = np.empty(len(out_steps) * len(components) * st.N, dtype=dtype)
        st.set_snapshots([comp_index(c) for c in components], out_steps, buf)
        stops = [Nt]
    else:
        stops = sorted(set(out_steps) | {Nt})
    a = 1
    for stop in stops:
        while a <= stop:
            b = min(stop, a + max_chunk - 1)
            try:
                st.run(a, b)
            except _abi.StepperError as e:
                if e.code == _abi.MFD_ERR_NONFINITE:
                    raise RuntimeError(str(e)) from None
                raise
            a = b + 1
        if stop in out_steps and not device_frames:
            for c in components:
                snaps[c].append(st.read_field(comp_index(c)).reshape(shape, order="F"))
            if "rho" in snaps:
                snaps["rho"].append(st.read_integral(_abi.MFD_INT_RHO).reshape(shape, order="F").astype(dtype))
    if device_frames:
        frames = buf.reshape(len(out_steps), len(components), st.N)
        for k, c in enumerate(components):
            snaps[c] = [frames[f, k].reshape(shape, order="F").copy() for f in range(len(out_steps))]
        st.set_snapshots([comp_index(components[0])], [], np.empty(0, dtype))
    if isfields:
        out["fields/t"] = np.asarray(t_T)[np.array(out_steps) - 1]
        for c, v in snaps.items():
            out["fields/" + c] = np.stack(v, axis=-1)
    out["Sa"] = st.read_integral(_abi.MFD_INT_SA).reshape(shape, order="F")
    if isgeometry:
        out["E2"] = st.read_integral(_abi.MFD_INT_E2).reshape(shape, order="F")
        if model.isplasma:
            out["rho_end"] = st.read_integral(_abi.MFD_INT_RHO).reshape(shape, order="F")
            out["JE"] = st.read_integral(_abi.MFD_INT_JE).reshape(shape, order="F")
    for n, ms in enumerate(meta["monitors"], start=1):
        cells = ms["cells"]
        pre = f"monitors/{n}/"
        out[pre + "issum"] = ms["sum"]
        out[pre + "inds"] = _cartesian(g, cells)
        spectral = ms["kind"] == 1
        if spectral:
            out[pre + "w"] = ms["dft"].w
        for c in comps_all:
            if spectral:
                shp = (ms["dft"].Nw,) if ms["sum"] else (ms["dft"].Nw, len(cells))
            else:
                shp = (Nt,) if ms["sum"] else (Nt, len(cells))
            v = st.read_monitor(n - 1, comp_index(c), shp, spectral)
            out[pre + c] = v if ms["sum"] else v.T
    fields = {c: st.read_field(comp_index(c)).reshape(shape, order="F")
              for c in field_components(g.ndim, model.polarization)}
    if tfsf_record:
        _, i1, i2 = meta["record"]
        rec = _record_dataset(g, st, meta, i1, i2, model.polarization)
        if tfsf_fname is None:
            base = fname if fname is not None else "out.npz"
            root, ext = os.path.splitext(base)
            tfsf_fname = root + "_tfsf" + (ext or ".npz")
        out["tfsf_record"] = rec
        d = os.path.dirname(tfsf_fname)
        if d:
            os.makedirs(d, exist_ok=True)
        np.savez(tfsf_fname, **rec)
        out["tfsf_fname"] = tfsf_fname
    if fname is not None:
        d = os.path.dirname(fname)
        if d:
            os.makedirs(d, exist_ok=True)
        saved = {k: v for k, v in out.items() if isinstance(v, (np.ndarray, bool, np.bool_, int, float))}
        if os.path.splitext(fname)[1].lower() in (".hdf", ".h5", ".hdf5"):
            write_hdf5(fname, saved)
        else:
            np.savez(fname, **saved)
    return Solution(model, Field(fields), out, np.asarray(t_T), np.dtype(dtype))


def write_hdf5(fname, out):
    """The reference's output file (outputs.jl, monitors.jl write_monitor) in HDF5: each
    "a/b/c" key a dataset c in group a/b.  The arrays here have the reference's Julia shapes
    (column-major, x fastest); HDF5.jl stores such an array with its dimensions reversed and
    its bytes unchanged, which is what transposing a column-major view to C order gives."""
    from . import hdf5
    tree = {}
    for key, v in out.items():
        parts = key.split("/")
        node = tree
        for p in parts[:-1]:
            node = node.setdefault(p, {})
        node[parts[-1]] = np.asarray(v).T
    hdf5.write(fname, tree)


def _cartesian(grid, cells):
    cells = np.asarray(cells, dtype=np.int64)
    if grid.ndim == 1:
        return (cells + 1)[:, None]
    if grid.ndim == 2:
        return np.stack([cells % grid.Nx + 1, cells // grid.Nx + 1], axis=1)
    return np.stack([cells % grid.Nx + 1, (cells // grid.Nx) % grid.Ny + 1,
                     cells // (grid.Nx * grid.Ny) + 1], axis=1)


def _record_dataset(g, st, meta, i1, i2, polarization="Hy"):
    """The TFSF record file content (sources.jl:349-369, 500-531, 779-836); the second 2-D
    field set records its faces over the nodes i1..i2."""
    box, _, _ = meta["record"]
    cs = meta["coords_T"]
    t_T = meta["t_T"]
    nt = len(t_T)
    rec = {"t": np.asarray(t_T), "box": np.asarray(box)}
    ix1, iy1, iz1 = i1
    ix2, iy2, iz2 = i2
    if g.ndim == 2:
        e = 1 if polarization == "Ey" else 0
        rec["x"] = np.asarray(cs[0][ix1 - 1:ix2 - 1 + e])
        rec["z"] = np.asarray(cs[1][iz1 - 1:iz2 - 1 + e])
    elif g.ndim == 3:
        rec["x"] = np.asarray(cs[0][ix1 - 1:ix2])
        rec["y"] = np.asarray(cs[1][iy1 - 1:iy2])
        rec["z"] = np.asarray(cs[2][iz1 - 1:iz2])
    Nxi, Nyi, Nzi = ix2 - ix1, iy2 - iy1, iz2 - iz1
    for k, name in enumerate(tfsf_names(g.ndim, polarization)):
        v = st.read_tfsf_record(k)
        if g.ndim == 1:
            rec[name] = v.reshape(nt)
        elif g.ndim == 2:
            rec[name] = v.reshape(nt, -1)
        else:
            face, j = k // 4, k % 4
            if face < 2:
                a, bb = (Nyi + 1, Nzi) if j in (0, 3) else (Nyi, Nzi + 1)
            elif face < 4:
                a, bb = (Nxi + 1, Nzi) if j in (0, 3) else (Nxi, Nzi + 1)
            else:
                a, bb = (Nxi + 1, Nyi) if j in (0, 3) else (Nxi, Nyi + 1)
            rec[name] = v.reshape(nt, bb, a)
    return rec
