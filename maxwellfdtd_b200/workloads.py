"""Synthetic workloads of the benchmark configurations, built through the public API.

plasmonics_256: 256^3 grid, dx = 2 nm, 12-cell CPML, a gold-like sphere (radius 60 nm,
eps_inf = 9, Drude wp = 1.37e16 rad/s, gamma = 1.07e14 1/s, one Lorentz pole deps = 1.1,
w0 = 4.2e15 rad/s, gamma = 1.0e15 1/s i.e. delta = gamma/2), an x-polarised broadband TFSF
plane wave along +z (600 nm, 3 fs), and DFT monitors on the six faces of a 160^3 box at 64
wavelengths 400-900 nm with double-precision sums.  The incident TFSF data are the
analytic plane wave sampled at the Yee positions, standing in for a vacuum record run.

plain_256: the plain FP32 stepper at 256^3 -- vacuum, dx = 2 nm, 12-cell CPML on all faces,
one soft point source; only the H/E updates with CPML and the Sa running sum.

batch2d: many independent 2-D models of seeded, uneven sizes -- Nx, Nz uniform in
[128, 1024], dx = 20 nm, 10-cell CPML, 2000-6000 steps (scaled by steps_scale), 1-20 random
ellipses per domain with eps uniform in [1, 12] and, for half of them, a Debye pole
(deps uniform in [1, 5], tau log-uniform in [1e-15, 1e-13] s), a soft Ricker point source
(lambda0 uniform in 400-1600 nm) and 4 point field monitors.

nonlinear_192: 192 x 192 x 1024 grid, dx = dy = 100 nm, dz = 20 nm, 16-cell CPML, FP32 with the
plasma density in FP64; the whole domain is a fused-silica-like glass: eps_inf = 1 and three
Lorentz poles from Malitson's Sellmeier fit (deps = B_i, w0 = 2 pi c / sqrt(C_i), small
damping), Kerr n2 = 2.5e-20 m^2/W (chi3 = 4/3 n0^2 eps0 c n2), an 8-photon ionisation
plasma (rate sigma8 I^8 with sigma8 = 1e-130, rho0 = 2.1e28 m^-3, collision time 1 fs,
Ui = 9 eV); a soft Gaussian-beam source (w0 = 3 um, 800 nm, 30 fs, 5e17 W/m^2) on a plane
near the low-z face.

served: a stream of solves of mixed kind for the serving loop -- Poisson arrivals; 2-D
(sides uniform in [256, 2048]) or 3-D (sides uniform in [64, 256]) grids, 500-5000 steps
(scaled by steps_scale); a random mix of dielectric, Drude and Lorentz spheres/discs; an
x-polarised plane-wave TFSF source (2-D) or a soft plane source; spectral monitors at 8-32
frequencies with FP64 sums on a line (2-D) or plane (3-D).

dielectric_100: 100^3 grid, dx = 20 nm, 10-cell CPML, Float64, a dielectric sphere
(radius 500 nm, eps = 2.25), a TFSF x-polarised Gaussian pulse (800 nm, 10 fs intensity
FWHM) along +z, and one point monitor.
"""
import numpy as np

from . import (C0, EPS0, MU0, Grid, DebyeSusceptibility, DrudeSusceptibility, FieldMonitor, LorentzSusceptibility,
               Material, Model, SeparableWaveform, SoftSource, SpectralMonitor, TFSFSource)
from .model import time_range, time_step
from .sources import TFSF_NAMES_3D


def _plane_wave_tfsf(grid, i1, i2, t, f, zs, dt):
    """TFSF record data of an x-polarised plane wave along +z: Ex = f(t - (z - zs)/c),
    Hy = Ex/eta0 sampled half a cell up and half a step earlier."""
    eta0 = np.sqrt(MU0 / EPS0)
    (ix1, iy1, iz1), (ix2, iy2, iz2) = i1, i2
    Nxi, Nyi, Nzi = ix2 - ix1, iy2 - iy1, iz2 - iz1
    z = grid.z
    dz = grid.dz
    nt = len(t)
    te = t + dt          # E at the end of step it
    th = t + dt / 2      # H half a step earlier

    def Ex(zv):
        return f(te[:, None] - (zv[None, :] - zs) / C0)

    def Hy(zv):
        return f(th[:, None] - (zv[None, :] + dz / 2 - zs) / C0) / eta0

    d = {"t": np.asarray(t), "box": np.array([grid.x[ix1 - 1], grid.x[ix2 - 1], grid.y[iy1 - 1], grid.y[iy2 - 1],
                                              grid.z[iz1 - 1], grid.z[iz2 - 1]]),
         "x": grid.x[ix1 - 1:ix2], "y": grid.y[iy1 - 1:iy2], "z": grid.z[iz1 - 1:iz2]}
    zh = z[iz1 - 1:iz2 - 1]      # iz1 .. iz2-1
    zf = z[iz1 - 1:iz2]          # iz1 .. iz2
    # The wave depends on z and t only, so every array is given with its constant face axes
    # of extent 1 (the [nt][b][a] layout broadcast): [nt][b][1] on the x and y faces, whose
    # b axis is z, [nt][1][1] on the z faces, and the components the wave lacks as zeros.
    for name in TFSF_NAMES_3D:
        d[name] = np.zeros((nt, 1, 1), dtype=np.float32)
    for name in ("incHy_1yz", "incHy_2yz"):          # (Nyi+1, Nzi): z in iz1..iz2-1
        d[name] = Hy(zh).astype(np.float32)[:, :, None]
    for name in ("incEx_x1z", "incEx_x2z"):          # (Nxi, Nzi+1): z in iz1..iz2
        d[name] = Ex(zf).astype(np.float32)[:, :, None]
    d["incHy_xy1"] = Hy(z[iz1 - 2:iz1 - 1]).astype(np.float32)[:, :, None]
    d["incEx_xy1"] = Ex(z[iz1 - 1:iz1]).astype(np.float32)[:, :, None]
    d["incHy_xy2"] = Hy(z[iz2 - 1:iz2]).astype(np.float32)[:, :, None]
    d["incEx_xy2"] = Ex(z[iz2 - 1:iz2]).astype(np.float32)[:, :, None]
    return d


def plasmonics_256(nt=4000, n=256, with_monitors=True):
    dx = 2e-9
    L = (n - 1) * dx / 2
    grid = Grid(xmin=-L, xmax=L, Nx=n, ymin=-L, ymax=L, Ny=n, zmin=-L, zmax=L, Nz=n)
    r = 60e-9
    gold = Material(geometry=lambda x, y, z: x * x + y * y + z * z <= r * r, eps=9.0,
                    chi=[DrudeSusceptibility(wp=1.37e16, gamma=1.07e14),
                         LorentzSusceptibility(deps=1.1, w0=4.2e15, delta=0.5e15)])
    dt = time_step(grid, 0.5)
    t = time_range(dt, (nt - 0.5) * dt)
    tau = 3e-15
    t0 = 3 * tau
    w0 = 2 * np.pi * C0 / 600e-9
    f = lambda s: np.exp(-2 * np.log(2) * (s - t0) ** 2 / tau ** 2) * np.cos(w0 * (s - t0))
    m = max(4, round(20 * n / 256))          # TFSF box faces 20 cells in from the edges at 256^3
    i1, i2 = (m, m, m), (n + 1 - m, n + 1 - m, n + 1 - m)
    data = _plane_wave_tfsf(grid, i1, i2, t, f, grid.z[i1[2] - 1], dt)
    model = Model(grid, TFSFSource(data=data), tmax=(nt - 0.5) * dt, pml=12 * dx, material=gold)
    mons = None
    if with_monitors:
        h = round(80 * n / 256) * dx + dx / 2   # faces on grid planes (coordinates are odd multiples of dx/2)
        lam = np.linspace(400e-9, 900e-9, 64)
        w = 2 * np.pi * C0 / lam
        eps = dx / 2
        box = lambda a: (np.abs(a) <= h + eps)
        faces = [
            lambda x, y, z: (np.abs(x + h) < eps) & box(y) & box(z),
            lambda x, y, z: (np.abs(x - h) < eps) & box(y) & box(z),
            lambda x, y, z: (np.abs(y + h) < eps) & box(x) & box(z),
            lambda x, y, z: (np.abs(y - h) < eps) & box(x) & box(z),
            lambda x, y, z: (np.abs(z + h) < eps) & box(x) & box(y),
            lambda x, y, z: (np.abs(z - h) < eps) & box(x) & box(y),
        ]
        mons = [SpectralMonitor(fc, w=w) for fc in faces]
    return model, mons


def _plane_wave_tfsf_2d(grid, i1, i2, t, f, zs, dt):
    """2-D TFSF record data of an x-polarised plane wave along +z (the layout a record run
    writes: knots x, z and per face [nt][knots])."""
    eta0 = np.sqrt(MU0 / EPS0)
    ix1, iz1 = i1[0], i1[2]
    ix2, iz2 = i2[0], i2[2]
    z, dz = grid.z, grid.dz
    te = t + dt
    th = t + dt / 2
    Ex = lambda zv: f(te[:, None] - (np.asarray(zv)[None, :] - zs) / C0)
    Hy = lambda zv: f(th[:, None] - (np.asarray(zv)[None, :] + dz / 2 - zs) / C0) / eta0
    xk = grid.x[ix1 - 1:ix2]
    zk = z[iz1 - 1:iz2]
    nt = len(t)
    d = {"t": np.asarray(t), "box": np.array([grid.x[ix1 - 1], grid.x[ix2 - 1], z[iz1 - 1], z[iz2 - 1]]),
         "x": xk, "z": zk}
    d["incHy_1z"] = Hy(zk).astype(np.float32)
    d["incEz_1z"] = np.zeros((nt, 1), np.float32)     # [nt][1]: the same (zero) along the face
    d["incHy_2z"] = d["incHy_1z"]
    d["incEz_2z"] = d["incEz_1z"]
    d["incHy_x1"] = Hy(z[iz1 - 2:iz1 - 1]).astype(np.float32)   # [nt][1]: uniform along x
    d["incEx_x1"] = Ex(z[iz1 - 1:iz1]).astype(np.float32)
    d["incHy_x2"] = Hy(z[iz2 - 1:iz2]).astype(np.float32)
    d["incEx_x2"] = Ex(z[iz2 - 1:iz2]).astype(np.float32)
    return d


def served(n=64, rate=200.0, seed=0, steps_scale=1.0, frac3d=0.5, n2=(256, 2048), n3=(64, 256)):
    """List of (arrival_s, model, monitors) for the serving loop, arrivals in order."""
    rng = np.random.default_rng(seed)
    t_arr = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for i in range(n):
        three = rng.uniform() < frac3d
        nsteps = max(2, int(round(int(rng.integers(500, 5001)) * steps_scale)))
        nw = int(rng.integers(8, 33))
        lam = np.linspace(400e-9, 900e-9, nw)
        w = 2 * np.pi * C0 / lam
        kinds = rng.integers(0, 3, size=int(rng.integers(1, 4)))
        if three:
            nn = [int(rng.integers(n3[0], n3[1] + 1)) for _ in range(3)]
            dx = 10e-9
            L = [(k - 1) * dx / 2 for k in nn]
            grid = Grid(xmin=-L[0], xmax=L[0], Nx=nn[0], ymin=-L[1], ymax=L[1], Ny=nn[1], zmin=-L[2], zmax=L[2], Nz=nn[2])
            rmax = 0.25 * min(L)
            pos = lambda: [float(rng.uniform(-0.3, 0.3) * l) for l in L]
        else:
            nn = [int(rng.integers(n2[0], n2[1] + 1)) for _ in range(2)]
            dx = 10e-9
            L = [(k - 1) * dx / 2 for k in nn]
            grid = Grid(xmin=-L[0], xmax=L[0], Nx=nn[0], zmin=-L[1], zmax=L[1], Nz=nn[1])
            rmax = 0.25 * min(L)
            pos = lambda: [float(rng.uniform(-0.3, 0.3) * l) for l in L]
        dt = time_step(grid, 0.5)
        mats = []
        for k in kinds:
            c = pos()
            r = float(rng.uniform(0.2, 1.0) * rmax)
            if three:
                geo = (lambda c, r: (lambda x, y, z: (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r))(c, r)
            else:
                geo = (lambda c, r: (lambda x, z: (x - c[0]) ** 2 + (z - c[1]) ** 2 <= r * r))(c, r)
            if k == 0:
                mats.append(Material(geometry=geo, eps=float(rng.uniform(1.5, 12))))
            elif k == 1:
                mats.append(Material(geometry=geo, eps=float(rng.uniform(1, 9)),
                                     chi=DrudeSusceptibility(wp=float(rng.uniform(0.5e16, 1.5e16)), gamma=1.07e14)))
            else:
                mats.append(Material(geometry=geo, eps=float(rng.uniform(1, 4)),
                                     chi=LorentzSusceptibility(deps=float(rng.uniform(0.5, 3)), w0=float(rng.uniform(2e15, 6e15)),
                                                               delta=5e14)))
        lam0 = float(rng.uniform(500e-9, 800e-9))
        w0 = 2 * np.pi * C0 / lam0
        tau = 5e-15
        f = lambda s, w0=w0, tau=tau: np.exp(-2 * np.log(2) * (s - 3 * tau) ** 2 / tau ** 2) * np.cos(w0 * (s - 3 * tau))
        pml = 10 * dx
        m_in = 14
        if not three and rng.uniform() < 0.5:
            t = time_range(dt, (nsteps - 0.5) * dt)
            i1 = (m_in, 1, m_in)
            i2 = (nn[0] + 1 - m_in, 1, nn[1] + 1 - m_in)
            data = _plane_wave_tfsf_2d(grid, i1, i2, t, f, grid.z[i1[2] - 1], dt)
            src = TFSFSource(data=data)
        else:
            z0 = -L[-1] + (m_in + 2) * dx
            if three:
                src = SoftSource(geometry=lambda x, y, z, z0=z0: np.abs(z - z0) < dx / 2,
                                 waveform=SeparableWaveform(lambda x, y, z: np.ones_like(x), f), component="Ex")
            else:
                src = SoftSource(geometry=lambda x, z, z0=z0: np.abs(z - z0) < dx / 2,
                                 waveform=SeparableWaveform(lambda x, z: np.ones_like(x), f), component="Ex")
        zm = L[-1] - (m_in + 2) * dx
        if three:
            mon = SpectralMonitor(lambda x, y, z, zm=zm: np.abs(z - zm) < dx / 2, w=w)
        else:
            mon = SpectralMonitor(lambda x, z, zm=zm: np.abs(z - zm) < dx / 2, w=w)
        model = Model(grid, src, tmax=(nsteps - 0.5) * dt, pml=pml, material=mats)
        out.append((float(t_arr[i]), model, [mon]))
    return out


def nonlinear_192(nt=12000, n=(192, 192, 1024)):
    from .materials import Plasma, PowerLawRate
    nx, ny, nz = n
    dx, dz = 100e-9, 20e-9
    Lx, Ly, Lz = (nx - 1) * dx / 2, (ny - 1) * dx / 2, (nz - 1) * dz / 2
    grid = Grid(xmin=-Lx, xmax=Lx, Nx=nx, ymin=-Ly, ymax=Ly, Ny=ny, zmin=-Lz, zmax=Lz, Nz=nz)
    dt = time_step(grid, 0.5)
    sellmeier = ((0.6961663, 0.0684043e-6), (0.4079426, 0.1162414e-6), (0.8974794, 9.896161e-6))
    chi = [LorentzSusceptibility(deps=B, w0=2 * np.pi * C0 / lam, delta=1e12) for B, lam in sellmeier]
    n0 = 1.45
    chi3 = 4 / 3 * n0 ** 2 * EPS0 * C0 * 2.5e-20
    lam0 = 800e-9
    w0 = 2 * np.pi * C0 / lam0
    plasma = Plasma(ionrate=PowerLawRate(order=8, sigma=1e-130), rho0=2.1e28, nuc=1 / 1e-15, frequency=w0, Uiev=9.0,
                    mr=0.64)
    glass = Material(geometry=lambda x, y, z: np.ones_like(x, dtype=bool), eps=1.0, chi=chi, chi3=chi3, plasma=plasma)
    I0, tau, wb = 5e17, 30e-15, 3e-6
    E0 = np.sqrt(2 * I0 / (n0 * EPS0 * C0))
    t0 = 2 * tau
    pulse = lambda t: np.exp(-2 * np.log(2) * (t - t0) ** 2 / tau ** 2) * np.cos(w0 * (t - t0))
    zs = -Lz + (16 + 4) * dz
    src = SoftSource(geometry=lambda x, y, z: np.abs(z - zs) < dz / 2,
                     waveform=SeparableWaveform(lambda x, y, z: E0 * np.exp(-(x ** 2 + y ** 2) / wb ** 2), pulse),
                     component="Ex")
    pml = (16 * dx, 16 * dx, 16 * dx, 16 * dx, 16 * dz, 16 * dz)
    return Model(grid, src, tmax=(nt - 0.5) * dt, pml=pml, material=glass), None


def dielectric_100_record(nt=1000, n=100):
    """The dielectric_100 configuration with its TFSF data made the reference's way: a
    vacuum run with a soft Ex plane source, periodic in x and y, absorbing in z, records the
    incident fields on the box (returns the record model and a function that builds the
    scattering model from the recorded data)."""
    dx = 20e-9
    L = (n - 1) * dx / 2
    grid = Grid(xmin=-L, xmax=L, Nx=n, ymin=-L, ymax=L, Ny=n, zmin=-L, zmax=L, Nz=n)
    dt = time_step(grid, 0.5)
    fwhm = 10e-15
    t0 = 3 * fwhm
    w0 = 2 * np.pi * C0 / 800e-9
    f = lambda s: np.exp(-2 * np.log(2) * (s - t0) ** 2 / fwhm ** 2) * np.cos(w0 * (s - t0))
    zs = -L + 12 * dx
    src = SoftSource(geometry=lambda x, y, z: np.abs(z - zs) < dx / 2,
                     waveform=SeparableWaveform(lambda x, y, z: np.ones_like(x), f), component="Ex")
    record = Model(grid, src, tmax=(nt - 0.5) * dt, pml=(0, 0, 0, 0, 10 * dx, 10 * dx))
    m = 11
    box = (grid.x[m - 1], grid.x[n - m], grid.y[m - 1], grid.y[n - m], grid.z[m - 1], grid.z[n - m])

    def scatter(data):
        r = 500e-9
        mat = Material(geometry=lambda x, y, z: x * x + y * y + z * z <= r * r, eps=2.25)
        return Model(grid, TFSFSource(data=data), tmax=(nt - 0.5) * dt, pml=10 * dx, material=mat), \
            [FieldMonitor((0.0, 0.0, 0.0))]
    return record, box, scatter


def plain_256(nt=40, n=256):
    dx = 2e-9
    L = (n - 1) * dx / 2
    grid = Grid(xmin=-L, xmax=L, Nx=n, ymin=-L, ymax=L, Ny=n, zmin=-L, zmax=L, Nz=n)
    dt = time_step(grid, 0.5)
    w0 = 2 * np.pi * C0 / 600e-9
    src = SoftSource(geometry=(0.0, 0.0, 0.0), waveform=lambda x, y, z, t: np.sin(w0 * t), component="Ex")
    return Model(grid, src, tmax=(nt - 0.5) * dt, pml=12 * dx), None


def dielectric_100(nt=1000, n=100):
    dx = 20e-9
    L = (n - 1) * dx / 2
    grid = Grid(xmin=-L, xmax=L, Nx=n, ymin=-L, ymax=L, Ny=n, zmin=-L, zmax=L, Nz=n)
    r = 500e-9
    mat = Material(geometry=lambda x, y, z: x * x + y * y + z * z <= r * r, eps=2.25)
    dt = time_step(grid, 0.5)
    t = time_range(dt, (nt - 0.5) * dt)
    fwhm = 10e-15
    t0 = 3 * fwhm
    w0 = 2 * np.pi * C0 / 800e-9
    f = lambda s: np.exp(-2 * np.log(2) * (s - t0) ** 2 / fwhm ** 2) * np.cos(w0 * (s - t0))
    m = 11
    i1, i2 = (m, m, m), (n + 1 - m, n + 1 - m, n + 1 - m)
    data = _plane_wave_tfsf(grid, i1, i2, t, f, grid.z[i1[2] - 1], dt)
    model = Model(grid, TFSFSource(data=data), tmax=(nt - 0.5) * dt, pml=10 * dx, material=mat)
    return model, [FieldMonitor((0.0, 0.0, 0.0))]


def ricker(lam0, ndim=2):
    """Ricker wavelet of centre frequency c/lam0, delayed by 1.5 periods (a waveform of the
    coordinates of an ndim-dimensional grid and t)."""
    f0 = C0 / lam0
    t0 = 1.5 / f0

    def r(t):
        a = (np.pi * f0 * (t - t0)) ** 2
        return (1 - 2 * a) * np.exp(-a)
    if ndim == 3:
        return lambda x, y, z, t: r(t)
    return lambda x, z, t: r(t)


def batch3d(n=64, seed=0, steps_scale=1.0, nmin=48, nmax=128):
    """List of (model, monitors) of small uneven 3-D models for a batch: sides uniform in
    [nmin, nmax] (independently per axis), dx = 20 nm, 8-cell CPML, 1-5 spheres with eps in
    [1, 12] (half of them Debye), a Ricker soft point source, 4 point monitors, 500-2000 steps."""
    rng = np.random.default_rng(seed)
    dx = 20e-9
    out = []
    for i in range(n):
        nn = [int(rng.integers(nmin, nmax + 1)) for _ in range(3)]
        nsteps = max(2, int(round(int(rng.integers(500, 2001)) * steps_scale)))
        L = [(k - 1) * dx / 2 for k in nn]
        grid = Grid(xmin=-L[0], xmax=L[0], Nx=nn[0], ymin=-L[1], ymax=L[1], Ny=nn[1], zmin=-L[2], zmax=L[2], Nz=nn[2])
        dt = time_step(grid, 0.5)
        mats = []
        for k in range(int(rng.integers(1, 6))):
            c = [float(rng.uniform(-0.6, 0.6) * l) for l in L]
            r = float(rng.uniform(0.05, 0.3) * min(L))
            geo = (lambda c, r: (lambda x, y, z: (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r))(c, r)
            eps = float(rng.uniform(1, 12))
            if rng.uniform() < 0.5:
                chi = DebyeSusceptibility(deps=float(rng.uniform(1, 5)), tau=float(10 ** rng.uniform(-15, -13)))
                mats.append(Material(geometry=geo, eps=eps, chi=chi))
            else:
                mats.append(Material(geometry=geo, eps=eps))
        lam0 = float(rng.uniform(400e-9, 1600e-9))
        sp = tuple(float(rng.uniform(-0.4, 0.4) * l) for l in L)
        src = SoftSource(geometry=sp, waveform=ricker(lam0, ndim=3), component="Ez")
        mons = [FieldMonitor(tuple(float(rng.uniform(-0.6, 0.6) * l) for l in L)) for _ in range(4)]
        model = Model(grid, src, tmax=(nsteps - 0.5) * dt, pml=8 * dx, material=mats)
        out.append((model, mons))
    return out


def batch2d(n=256, seed=0, steps_scale=1.0, nmin=128, nmax=1024):
    """List of (model, monitors) for the batched 2-D configuration."""
    rng = np.random.default_rng(seed)
    dx = 20e-9
    out = []
    for i in range(n):
        nx, nz = int(rng.integers(nmin, nmax + 1)), int(rng.integers(nmin, nmax + 1))
        nsteps = max(2, int(round(int(rng.integers(2000, 6001)) * steps_scale)))
        Lx, Lz = (nx - 1) * dx / 2, (nz - 1) * dx / 2
        grid = Grid(xmin=-Lx, xmax=Lx, Nx=nx, zmin=-Lz, zmax=Lz, Nz=nz)
        dt = time_step(grid, 0.5)
        mats = []
        for k in range(int(rng.integers(1, 21))):
            cx, cz = rng.uniform(-0.8, 0.8) * Lx, rng.uniform(-0.8, 0.8) * Lz
            a, b = rng.uniform(0.02, 0.25) * Lx, rng.uniform(0.02, 0.25) * Lz
            geo = (lambda cx, cz, a, b: (lambda x, z: ((x - cx) / a) ** 2 + ((z - cz) / b) ** 2 <= 1))(cx, cz, a, b)
            eps = float(rng.uniform(1, 12))
            if rng.uniform() < 0.5:
                chi = DebyeSusceptibility(deps=float(rng.uniform(1, 5)), tau=float(10 ** rng.uniform(-15, -13)))
                mats.append(Material(geometry=geo, eps=eps, chi=chi))
            else:
                mats.append(Material(geometry=geo, eps=eps))
        lam0 = float(rng.uniform(400e-9, 1600e-9))
        sx, sz = rng.uniform(-0.5, 0.5) * Lx, rng.uniform(-0.5, 0.5) * Lz
        src = SoftSource(geometry=(sx, sz), waveform=ricker(lam0), component="Ez")
        mons = [FieldMonitor((float(rng.uniform(-0.7, 0.7) * Lx), float(rng.uniform(-0.7, 0.7) * Lz))) for _ in range(4)]
        model = Model(grid, src, tmax=(nsteps - 0.5) * dt, pml=10 * dx, material=mats)
        out.append((model, mons))
    return out

