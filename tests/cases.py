"""Small models that exercise every part of the time-step path, built through the public
Python API, plus a runner that executes one model on a given library and collects every
output (fields incl. D, Sa, E2, JE, rho_end, monitors, TFSF record)."""
import numpy as np

import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import C0, EPS0, _abi
from maxwellfdtd_b200.sources import comp_index, field_components


def pulse(t, lam0=1e-6, tau0=4e-15, t0=None):
    t0 = 3 * tau0 if t0 is None else t0
    w0 = 2 * np.pi * C0 / lam0
    return np.exp(-(t - t0) ** 2 / tau0 ** 2) * np.cos(w0 * (t - t0))


def grid3(n=(20, 18, 16), d=50e-9):
    nx, ny, nz = n
    return M.Grid(xmin=-(nx - 1) * d / 2, xmax=(nx - 1) * d / 2, Nx=nx,
                  ymin=-(ny - 1) * d / 2, ymax=(ny - 1) * d / 2, Ny=ny,
                  zmin=-(nz - 1) * d / 2, zmax=(nz - 1) * d / 2, Nz=nz)


def grid2(n=(24, 30), d=50e-9):
    nx, nz = n
    return M.Grid(xmin=-(nx - 1) * d / 2, xmax=(nx - 1) * d / 2, Nx=nx,
                  zmin=-(nz - 1) * d / 2, zmax=(nz - 1) * d / 2, Nz=nz)


def grid1(n=80, d=50e-9):
    return M.Grid(zmin=-(n - 1) * d / 2, zmax=(n - 1) * d / 2, Nz=n)


def _geo_point(ndim, where=(0.0, 0.0, 0.0)):
    return tuple(where[:ndim]) if ndim == 3 else ((where[0], where[2]) if ndim == 2 else (where[2],))


def _src_wave(ndim, amp=1.0, lam0=1e-6):
    if ndim == 3:
        return lambda x, y, z, t: amp * np.exp(-(x ** 2 + y ** 2) / (300e-9) ** 2) * pulse(t, lam0)
    if ndim == 2:
        return lambda x, z, t: amp * np.exp(-(x ** 2) / (300e-9) ** 2) * pulse(t, lam0)
    return lambda z, t: amp * pulse(t, lam0)


def _plane(ndim, z0):
    if ndim == 3:
        return lambda x, y, z: np.abs(z - z0) < 26e-9
    if ndim == 2:
        return lambda x, z: np.abs(z - z0) < 26e-9
    return lambda z: np.abs(z - z0) < 26e-9


def _ball(ndim, r, c=(0.0, 0.0, 0.0)):
    if ndim == 3:
        return lambda x, y, z: (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r
    if ndim == 2:
        return lambda x, z: (x - c[0]) ** 2 + (z - c[2]) ** 2 <= r * r
    return lambda z: np.abs(z - c[2]) <= r


def _grid(ndim):
    return grid3() if ndim == 3 else grid2() if ndim == 2 else grid1()


def model_vacuum(ndim, nsteps=60):
    g = _grid(ndim)
    src = M.SoftSource(geometry=_plane(ndim, -200e-9), waveform=_src_wave(ndim), component="Ex")
    dt = 0.5 / C0 / np.sqrt(ndim / (50e-9) ** 2)
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=150e-9)


def model_bcs(ndim, nsteps=60):
    """Mixed boundary conditions, CPML with kmax != 1 on some faces and none on others."""
    g = _grid(ndim)
    src = M.SoftSource(geometry=_geo_point(ndim, (50e-9, 0.0, -100e-9)), waveform=_src_wave(ndim, 3.0),
                       component="Ez" if ndim > 1 else "Ex")
    dt = 0.5 / C0 / np.sqrt(ndim / (50e-9) ** 2)
    cp = M.CPML(thickness=150e-9, kmax=4.0, alpha=0.05, R0=1e-8, m=4)
    if ndim == 3:
        bc = ("periodic", "dirichlet", "neumann", "periodic", "dirichlet", "neumann")
        pml = (cp, 0, 100e-9, cp, 0, cp)
    elif ndim == 2:
        bc = ("dirichlet", "neumann", "periodic", "periodic")
        pml = (0, cp, cp, 0)
    else:
        bc = ("neumann", "dirichlet")
        pml = (cp, 0)
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=pml, bc=bc)


def model_materials(ndim, nsteps=70):
    """Conductive dielectric with mu != 1, Drude+Lorentz ball, Debye+Kerr slab; later
    materials overwrite earlier ones."""
    g = _grid(ndim)
    src = M.SoftSource(geometry=_plane(ndim, -250e-9), waveform=_src_wave(ndim, 2e8), component="Ex")
    dt = 0.5 / C0 / np.sqrt(ndim / (50e-9) ** 2)
    if ndim == 3:
        slab = lambda x, y, z: z >= 150e-9
        half = lambda x, y, z: x > 0
    elif ndim == 2:
        slab = lambda x, z: z >= 150e-9
        half = lambda x, z: x > 0
    else:
        slab = lambda z: z >= 250e-9
        half = lambda z: z > 300e-9
    m1 = M.Material(geometry=half, eps=2.25, mu=1.3, sigma=2e4)
    m2 = M.Material(geometry=_ball(ndim, 160e-9), eps=3.0,
                    chi=[M.DrudeSusceptibility(wp=1.37e16, gamma=1.07e14),
                         M.LorentzSusceptibility(deps=1.1, w0=4.2e15, delta=5e14)])
    m3 = M.Material(geometry=slab, eps=2.0, chi=M.DebyeSusceptibility(deps=2.0, tau=1e-14), chi3=1e-19, chi2=1e-12)
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=150e-9, material=[m1, m2, m3])


def model_plasma(ndim, rate="power", nsteps=60):
    g = _grid(ndim)
    E0 = 1.3e10
    src = M.SoftSource(geometry=_plane(ndim, -250e-9), waveform=_src_wave(ndim, E0), component="Ex")
    dt = 0.5 / C0 / np.sqrt(ndim / (50e-9) ** 2)
    w0 = 2 * np.pi * C0 / 800e-9
    if rate == "power":
        ionrate = M.PowerLawRate(order=8, sigma=1e-130)
    else:
        I = np.logspace(12, 20, 81)
        ionrate = M.IonizationRate(np.stack([I, 1e-130 * I ** 8], axis=1))
    pl = M.Plasma(ionrate=ionrate, rho0=2.1e28, nuc=1 / 1e-15, frequency=w0, Uiev=9.0, mr=0.64)
    chi3 = 4 / 3 * 1.45 ** 2 * EPS0 * C0 * 2.5e-20
    mat = M.Material(geometry=_ball(ndim, 250e-9), eps=1.45 ** 2, chi3=chi3, plasma=pl,
                     chi=M.LorentzSusceptibility(deps=0.7, w0=1.6e16, delta=1e13))
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=150e-9, material=mat)


def model_sources(ndim, nsteps=50):
    """Hard source on H, explicit soft source on E, soft source on D (tuple order)."""
    g = _grid(ndim)
    dt = 0.5 / C0 / np.sqrt(ndim / (50e-9) ** 2)
    s1 = M.HardSource(geometry=_geo_point(ndim, (0.0, 0.0, -150e-9)), waveform=_src_wave(ndim, 1e-3), component="Hy")
    s2 = M.SoftSource(geometry=_plane(ndim, 100e-9), waveform=_src_wave(ndim, 0.7), component="Ex", explicit=True)
    s3 = M.SoftSource(geometry=_plane(ndim, 100e-9), waveform=_src_wave(ndim, 0.3), component="Ex")
    return M.Model(g, [s1, s2, s3], tmax=(nsteps - 0.5) * dt, pml=100e-9)


def model_wide_rows(bcx, nsteps=45):
    """3-D rows longer than one warp's span of 4-cell groups and not a multiple of 4 cells
    (137 x 5 x 6): sources on the first and the last x cell so the x boundary condition
    matters, CPML on the left x face, materials straddling group and warp boundaries."""
    g = grid3((137, 5, 6))
    xe = 68 * 50e-9
    src = M.SoftSource(geometry=lambda x, y, z: np.abs(x - xe) < 26e-9,
                       waveform=lambda x, y, z, t: 1e3 * pulse(t), component="Ez")
    s2 = M.SoftSource(geometry=(-xe, 0.0, 0.0), waveform=lambda x, y, z, t: 5e2 * pulse(t), component="Ey")
    dt = 0.5 / C0 / np.sqrt(3 / (50e-9) ** 2)
    m1 = M.Material(geometry=lambda x, y, z: x > 0.3e-6, eps=2.25, mu=1.3, sigma=2e4)
    m2 = M.Material(geometry=lambda x, y, z: np.abs(x + 0.2e-6) < 130e-9, eps=3.0,
                    chi=M.DrudeSusceptibility(wp=1.37e16, gamma=1.07e14))
    return M.Model(g, [src, s2], tmax=(nsteps - 0.5) * dt, pml=(150e-9, 0, 0, 0, 0, 0),
                   bc=(bcx, bcx, "periodic", "periodic", "neumann", "dirichlet"), material=[m1, m2])


def model_layers(n, pml, nsteps=40):
    """3-D grid of n cells with the given CPML thicknesses (faces xl, xr, yl, yr, zl, zr),
    e.g. layers that overlap in a dimension or exist on one axis only."""
    g = grid3(n)
    src = M.SoftSource(geometry=(0.0, 0.0, 0.0), waveform=lambda x, y, z, t: 1e3 * pulse(t), component="Ez")
    dt = 0.5 / C0 / np.sqrt(3 / (50e-9) ** 2)
    m1 = M.Material(geometry=lambda x, y, z: x + y > 0, eps=2.25, mu=1.3, sigma=2e4)
    cp = M.CPML(thickness=150e-9, kmax=3.0, alpha=0.05, R0=1e-8, m=3)
    faces = tuple(cp if t else 0 for t in pml)
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=faces, material=m1)


def model_poles(ndim, npoles, kerr=False, nsteps=50):
    """A ball with npoles dispersion poles (Lorentz/Drude/Debye in turn), optionally Kerr,
    overlapping a slab with one pole: the material kernels by pole count."""
    g = _grid(ndim)
    src = M.SoftSource(geometry=_plane(ndim, -250e-9), waveform=_src_wave(ndim, 3e8), component="Ex")
    dt = 0.5 / C0 / np.sqrt(ndim / (50e-9) ** 2)
    kinds = [lambda i: M.LorentzSusceptibility(deps=0.5 + 0.2 * i, w0=(3 + i) * 1e15, delta=(1 + i) * 1e14),
             lambda i: M.DrudeSusceptibility(wp=(1 + 0.1 * i) * 1e16, gamma=1.07e14),
             lambda i: M.DebyeSusceptibility(deps=1.0 + i, tau=(1 + i) * 1e-14)]
    chi = [kinds[i % 3](i) for i in range(npoles)]
    m1 = M.Material(geometry=_ball(ndim, 200e-9), eps=2.0, chi=chi, chi3=1e-19 if kerr else None)
    slab = (lambda x, y, z: z >= 200e-9) if ndim == 3 else ((lambda x, z: z >= 200e-9) if ndim == 2 else (lambda z: z >= 300e-9))
    m2 = M.Material(geometry=slab, eps=1.5, chi=M.LorentzSusceptibility(deps=0.7, w0=5e15, delta=2e14))
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=150e-9, material=[m1, m2])


def monitors(ndim):
    pt = _geo_point(ndim, (0.0, 0.0, 100e-9))
    plane = _plane(ndim, 150e-9)
    return [M.FieldMonitor(pt), M.FieldMonitor(plane, sum=True), M.FieldMonitor(plane),
            M.SpectralMonitor(plane, wmin=1e15, wmax=4e15),
            M.SpectralMonitor(plane, sum=True),
            M.SpectralMonitor(pt, w=np.linspace(1.2e15, 3.2e15, 11))]


def tfsf_box(ndim):
    h = 250e-9
    if ndim == 3:
        return (-h, h, -h, h, -h, h)
    if ndim == 2:
        return (-h, h, -h, h)
    return (-h, h)


def model_tfsf_record(ndim, nsteps=60):
    """Vacuum record run: plane source, periodic in x/y, absorbing in z (sources.jl:779-877)."""
    g = _grid(ndim)
    src = M.SoftSource(geometry=_plane(ndim, -400e-9 if ndim < 3 else -300e-9),
                       waveform=(lambda x, y, z, t: pulse(t)) if ndim == 3 else
                       (lambda x, z, t: pulse(t)) if ndim == 2 else (lambda z, t: pulse(t)),
                       component="Ex")
    dt = 0.5 / C0 / np.sqrt(ndim / (50e-9) ** 2)
    pml = (0, 0, 0, 0, 100e-9, 100e-9) if ndim == 3 else (0, 0, 100e-9, 100e-9) if ndim == 2 else 100e-9
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=pml)


def model_tfsf_replay(ndim, record, nsteps=60):
    g = _grid(ndim)
    dt = 0.5 / C0 / np.sqrt(ndim / (50e-9) ** 2)
    src = M.TFSFSource(data=record)
    mat = M.Material(geometry=_ball(ndim, 120e-9), eps=2.25)
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=100e-9, material=mat)


def run_all(model, library, dtype, mons=None, tfsf_box_=None, rho_fp64=True, chunks=None, mode="exact"):
    """Run a model on a library; return a dict of every output array."""
    be = M.B200(dtype, library=library, rho_fp64=rho_fp64, mode=mode)
    if chunks is None:
        sol = M.solve(model, backend=be, monitors=mons, tfsf_record=tfsf_box_ is not None, tfsf_box=tfsf_box_,
                      tfsf_fname=None if tfsf_box_ is None else _tmp_name())
        out = {f"field/{c}": np.asarray(sol.field[c]) for c in field_components(model.grid.ndim, model.polarization)}
        for k, v in sol.out.items():
            if isinstance(v, np.ndarray) and k != "t":
                out[k] = v
        if "tfsf_record" in sol.out:
            for k, v in sol.out["tfsf_record"].items():
                out["rec/" + k] = np.asarray(v)
        return out
    # chunked driving straight through the ABI
    b, meta = model.build_desc(dtype, mons, rho_fp64=rho_fp64, mode=mode)
    st = _abi.Stepper(library, b, dtype)
    a = 1
    for n in chunks:
        st.run(a, a + n - 1)
        a += n
    st.run(a, model.Nt)
    out = {f"field/{c}": st.read_field(comp_index(c)) for c in field_components(model.grid.ndim, model.polarization)}
    out["Sa"] = st.read_integral(_abi.MFD_INT_SA)
    st.close()
    return out


_TMP = [0]


def _tmp_name():
    import os
    import tempfile
    _TMP[0] += 1
    return os.path.join(tempfile.gettempdir(), f"mfd_rec_{os.getpid()}_{_TMP[0]}.npz")
